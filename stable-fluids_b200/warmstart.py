"""The learned pressure warm start, driven through the C ABI
(stable_fluids_b200_network_* in include/stable-fluids-b200.h).

`WarmStartNetwork` owns one network object of the library: a 3-level 3D U-Net
(16/32/64 channels) whose forward pass, backward pass and Adam step all run
in the library's own CUDA kernels (implicit-GEMM 3x3x3 convolutions on the
tensor cores, BF16 weights/activations, FP32 accumulation). torch only
provides device buffers and the stream handle.

`training_pairs` produces (b, p_prev, p_target) triples from a running
simulation: it steps a context stage by stage, snapshots the pressure
right-hand side (the pre-projection divergence) and the previous pressure
before the pressure solve, and takes the solved pressure (a long Jacobi
solve) as the target.
"""

from __future__ import annotations

import ctypes
import pathlib
from ctypes import byref, c_double, c_uint64, c_void_p

import numpy as np

from . import (
    RESULT_OK,
    STAGE_DIAGNOSTICS,
    STAGE_DIVERGENCE,
    STAGE_FORCES,
    STAGE_PRESSURE,
    STAGE_PROJECTION,
    STAGE_SCALARS,
    STAGE_VELOCITY_ADVECTION,
    STAGE_VELOCITY_DIFFUSION,
    VIEW_FLOW_DIVERGENCE,
    VIEW_FLOW_PRESSURE,
    load_library,
)

# (name, cin, cout) in forward order, padded channel counts; the parameter
# vector holds per layer weights [27][cout][cin] then cout biases.
LAYERS = (
    ("enc0a", 16, 16), ("enc0b", 16, 16), ("enc1a", 16, 32), ("enc1b", 32, 32),
    ("bott_a", 32, 64), ("bott_b", 64, 64), ("dec1a", 96, 32), ("dec1b", 32, 32),
    ("dec0a", 48, 16), ("dec0b", 16, 16), ("out", 16, 16),
)


def parameter_count() -> int:
    return sum(27 * ci * co + co for _, ci, co in LAYERS)


def split_parameters(flat: np.ndarray) -> dict[str, tuple[np.ndarray, np.ndarray]]:
    """Views of a flat parameter vector as {layer: (w[27, cout, cin], b[cout])}."""
    out, off = {}, 0
    for name, ci, co in LAYERS:
        wn = 27 * ci * co
        out[name] = (flat[off:off + wn].reshape(27, co, ci), flat[off + wn:off + wn + co])
        off += wn + co
    return out


class WarmStartNetwork:
    def __init__(self, seed: int = 0, *, lib=None, device: int = 0):
        import torch

        self._torch = torch
        self.lib = lib if lib is not None else load_library()
        self.device = torch.device("cuda", device)
        h = c_void_p()
        with torch.cuda.device(self.device):
            rc = self.lib.stable_fluids_b200_network_create(seed, byref(h))
        if rc != RESULT_OK:
            raise RuntimeError(f"stable_fluids_b200_network_create failed ({rc})")
        self.handle = h
        self.stream = torch.cuda.Stream(device=self.device)

    # --------------------------------------------------------- parameters --
    def parameters(self) -> np.ndarray:
        n = c_uint64(0)
        self._check(self.lib.stable_fluids_b200_network_parameters(self.handle, byref(n), None), "network_parameters")
        out = np.empty(n.value, dtype=np.float32)
        self._check(self.lib.stable_fluids_b200_network_parameters(self.handle, None, out.ctypes.data_as(c_void_p)), "network_parameters")
        return out

    def set_parameters(self, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float32)
        if a.size != parameter_count():
            raise ValueError(f"{a.size} parameters given, the network has {parameter_count()}")
        self._check(self.lib.stable_fluids_b200_network_set_parameters(self.handle, a.ctypes.data_as(c_void_p)), "network_set_parameters")

    def save(self, path: str | pathlib.Path):
        np.save(path, self.parameters())

    def load(self, path: str | pathlib.Path):
        self.set_parameters(np.load(path))

    # ------------------------------------------------------------ compute --
    def _dev(self, a):
        torch = self._torch
        if a is None:
            return None
        if isinstance(a, torch.Tensor):
            return a.to(self.device, torch.float32).contiguous()
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(self.device)

    @staticmethod
    def _ptr(t):
        return None if t is None else t.data_ptr()

    def predict(self, b, p_prev, cell_size: float):
        """Warm-start pressure (torch tensor, shape of b) from the divergence b
        and the previous pressure (None = zero)."""
        torch = self._torch
        bd, pd = self._dev(b), self._dev(p_prev)
        out = torch.empty_like(bd)
        nz, ny, nx = bd.shape
        torch.cuda.current_stream(self.device).synchronize()
        self._check(self.lib.stable_fluids_b200_network_predict(self.handle, self._ptr(bd), self._ptr(pd), nx, ny, nz, cell_size, self._ptr(out), c_void_p(self.stream.cuda_stream)), "network_predict")
        self.stream.synchronize()
        return out

    def gradients(self, b, p_prev, p_target, cell_size: float) -> tuple[float, np.ndarray]:
        """(loss, gradient of the loss w.r.t. every parameter)."""
        bd, pd, td = self._dev(b), self._dev(p_prev), self._dev(p_target)
        nz, ny, nx = bd.shape
        loss = c_double(0.0)
        g = np.empty(parameter_count(), dtype=np.float32)
        self._torch.cuda.current_stream(self.device).synchronize()
        self._check(self.lib.stable_fluids_b200_network_gradients(self.handle, self._ptr(bd), self._ptr(pd), self._ptr(td), nx, ny, nz, cell_size, byref(loss), g.ctypes.data_as(c_void_p), c_void_p(self.stream.cuda_stream)), "network_gradients")
        return loss.value, g

    def train_step(self, b, p_prev, p_target, cell_size: float, learning_rate: float) -> float:
        """One Adam step; returns the loss before it."""
        bd, pd, td = self._dev(b), self._dev(p_prev), self._dev(p_target)
        nz, ny, nx = bd.shape
        loss = c_double(0.0)
        self._torch.cuda.current_stream(self.device).synchronize()
        self._check(self.lib.stable_fluids_b200_network_train_step(self.handle, self._ptr(bd), self._ptr(pd), self._ptr(td), nx, ny, nz, cell_size, learning_rate, byref(loss), c_void_p(self.stream.cuda_stream)), "network_train_step")
        return loss.value

    def attach(self, simulation):
        """Uses this network for the warm start of a Simulation created with
        warm_start = LEARNED (rebuilds its step graph)."""
        self._check(self.lib.stable_fluids_b200_attach_network(simulation.ctx, self.handle), "attach_network")

    @staticmethod
    def detach(simulation):
        rc = simulation.lib.stable_fluids_b200_attach_network(simulation.ctx, None)
        if rc != RESULT_OK:
            raise RuntimeError(f"stable_fluids_b200_attach_network failed ({rc})")

    def _check(self, rc, what):
        if rc != RESULT_OK:
            raise RuntimeError(f"stable_fluids_b200_{what} failed ({rc})")

    def close(self):
        if getattr(self, "handle", None):
            self.lib.stable_fluids_b200_network_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def step_with_snapshot(sim):
    """One simulation step run stage by stage (the step graph's order) that
    returns (b, p_prev, p_solved) as device tensor copies: the pressure
    right-hand side's divergence and the pressure before and after the solve."""
    torch = sim._torch
    for stage in (STAGE_FORCES, STAGE_VELOCITY_ADVECTION, STAGE_VELOCITY_DIFFUSION, STAGE_DIVERGENCE):
        sim.enqueue_stage(stage)
    with torch.cuda.stream(sim.stream):
        div = sim.view(VIEW_FLOW_DIVERGENCE).clone()
        p_prev = sim.view(VIEW_FLOW_PRESSURE).clone()
    sim.enqueue_stage(STAGE_PRESSURE)
    with torch.cuda.stream(sim.stream):
        p_solved = sim.view(VIEW_FLOW_PRESSURE).clone()
    for stage in (STAGE_PROJECTION, STAGE_SCALARS, STAGE_DIAGNOSTICS):
        sim.enqueue_stage(stage)
    sim.stream.synchronize()
    return div, p_prev, p_solved


def training_pairs(make_simulation, steps: int, skip: int = 0):
    """Yields (b, p_prev, p_target) from `steps` stage-by-stage steps of the
    simulation `make_simulation()` returns (its pressure solve defines the
    target), after `skip` plain steps."""
    sim = make_simulation()
    try:
        sim.step(skip)
        for _ in range(steps):
            yield step_with_snapshot(sim)
    finally:
        sim.synchronize()
        sim.close()


def generate_pairs(sf, scene, steps: int, skip: int = 2, lib=None):
    """(b, p_prev, p_target) device tensors from `steps` steps of `scene`
    after `skip` plain ones, with the scene's pressure solve (Jacobi sweeps
    from the previous pressure) as the target generator."""
    def make():
        o = sf.default_options(lib)
        o.scheme = sf.SCHEME_JACOBI
        o.warm_start = sf.WARM_START_PREVIOUS
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib, options=o)
        sf.scenes.apply_inputs(sim, scene, 0)
        return sim

    return list(training_pairs(make, steps=steps, skip=skip))


def train(net, pairs, cell_size: float, epochs: int, learning_rate: float, seed: int = 0, deadline: float | None = None):
    """Adam over `pairs` in shuffled order for `epochs` epochs (or until the
    perf_counter `deadline`); returns the per-epoch mean losses."""
    import time

    rng = np.random.default_rng(seed)
    history = []
    for _ in range(epochs):
        order = rng.permutation(len(pairs))
        losses = []
        for k in order:
            b, p, t = pairs[k]
            losses.append(net.train_step(b, p, t, cell_size, learning_rate))
            if deadline is not None and time.perf_counter() > deadline:
                break
        history.append(float(np.mean(losses)))
        if deadline is not None and time.perf_counter() > deadline:
            break
    return history
