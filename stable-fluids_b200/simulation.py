"""`Simulation`: one stable-fluids context driven through the C ABI.

Field arrays are shaped (nz, ny, nx) -- x fastest, the ABI's dense layout.
Inputs may be numpy arrays (copied to the device on the simulation's stream
first, since the upstream ABI takes device pointers), CUDA torch tensors, or
None (zero-fill, as the ABI defines for a null pointer).
"""

from __future__ import annotations

import ctypes
import os
from ctypes import byref, c_uint32, c_void_p

import numpy as np

from . import (
    RESULT_OK,
    VIEW_FLOW_VELOCITY,
    VIEW_VECTOR_FIELD,
    B200Options,
    B200StepInfo,
    B200StepStats,
    ContextCreateDesc,
    ScalarFieldDesc,
    SimulationConfig,
    VectorFieldDesc,
    View,
    ViewRequest,
    load_library,
)


class StableFluidsError(RuntimeError):
    def __init__(self, what: str, code: int):
        super().__init__(f"{what} failed with StableFluidsResult {code}")
        self.code = code


class _DeviceArray:
    """Zero-copy handle on library-owned device memory for torch.as_tensor."""

    def __init__(self, ptr: int, shape: tuple[int, ...]):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (int(ptr), False), "version": 3, "strides": None, "stream": None}


class Simulation:
    def __init__(self, config: SimulationConfig, scalar_fields=(), vector_fields=(), *, lib=None, options: B200Options | None = None, device: int = 0):
        import torch

        self._torch = torch
        self.lib = lib if lib is not None else load_library()
        self.config = config
        self.shape = (config.nz, config.ny, config.nx)
        self.cells = config.nx * config.ny * config.nz
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(device=self.device)
        self._keep: list = []
        self._scalars = (ScalarFieldDesc * max(1, len(scalar_fields)))(*scalar_fields)
        self._vectors = (VectorFieldDesc * max(1, len(vector_fields)))(*vector_fields)
        desc = ContextCreateDesc(
            config=config,
            stream=c_void_p(self.stream.cuda_stream),
            scalar_fields=ctypes.cast(self._scalars, ctypes.POINTER(ScalarFieldDesc)),
            scalar_field_count=len(scalar_fields),
            vector_fields=ctypes.cast(self._vectors, ctypes.POINTER(VectorFieldDesc)),
            vector_field_count=len(vector_fields),
        )
        self._desc = desc
        hs = (c_uint32 * max(1, len(scalar_fields)))()
        hv = (c_uint32 * max(1, len(vector_fields)))()
        ctx = c_void_p()
        with torch.cuda.device(self.device):
            if options is not None:
                if not getattr(self.lib, "_sf_extended", False):
                    raise ValueError("this library has no stable_fluids_b200_create_context")
                rc = self.lib.stable_fluids_b200_create_context(byref(desc), byref(options), byref(ctx), hs, len(scalar_fields), hv, len(vector_fields))
            else:
                rc = self.lib.stable_fluids_create_context_cuda(byref(desc), byref(ctx), hs, len(scalar_fields), hv, len(vector_fields))
        if rc != RESULT_OK:
            raise StableFluidsError("stable_fluids_create_context", rc)
        self.ctx = ctx
        self.scalar_handles = [hs[i] for i in range(len(scalar_fields))]
        self.vector_handles = [hv[i] for i in range(len(vector_fields))]

    # ----------------------------------------------------------- inputs --
    def _device_ptr(self, values):
        if values is None:
            return None
        torch = self._torch
        if isinstance(values, torch.Tensor):
            t = values
            if t.device != self.device or t.dtype != torch.float32 or not t.is_contiguous():
                with torch.cuda.stream(self.stream):
                    t = t.to(self.device, torch.float32).contiguous()
        else:
            a = np.ascontiguousarray(values, dtype=np.float32)
            with torch.cuda.stream(self.stream):
                t = torch.from_numpy(a).to(self.device, non_blocking=False)
        if t.numel() != self.cells:
            raise ValueError(f"field has {t.numel()} values, grid has {self.cells}")
        self._keep.append(t)
        return t.data_ptr()

    def _check(self, rc: int, what: str):
        if rc != RESULT_OK:
            raise StableFluidsError(what, rc)

    def set_scalar(self, handle: int, values):
        self._check(self.lib.stable_fluids_update_scalar_field_cuda(self.ctx, handle, self._device_ptr(values)), "update_scalar_field")

    def set_scalar_source(self, handle: int, values):
        self._check(self.lib.stable_fluids_update_scalar_field_source_cuda(self.ctx, handle, self._device_ptr(values)), "update_scalar_field_source")

    def set_vector(self, handle: int, x, y, z):
        px, py, pz = self._device_ptr(x), self._device_ptr(y), self._device_ptr(z)
        self._check(self.lib.stable_fluids_update_vector_field_cuda(self.ctx, handle, px, py, pz), "update_vector_field")

    def stage_vector(self, handle: int, x, y, z, copy_stream):
        """Staged update (stable_fluids_b200_stage_vector_field): x, y, z are
        pinned host (or device) torch tensors of the grid's size, or None
        (zero); copied on `copy_stream` (a torch.cuda.Stream) and applied by
        the next step. Keep the tensors unchanged until the copy has run."""
        ptr = [None if t is None else c_void_p(t.data_ptr()) for t in (x, y, z)]
        self._check(self.lib.stable_fluids_b200_stage_vector_field(self.ctx, handle, ptr[0], ptr[1], ptr[2], c_void_p(copy_stream.cuda_stream)), "stage_vector_field")

    def read_view_async(self, kind: int, outs, copy_stream, handle: int = 0):
        """Asynchronous read-back (stable_fluids_b200_read_view_async) into
        pinned host tensors `outs` (one, or three for the vector layouts) on
        `copy_stream`; the data is there once copy_stream has passed it."""
        req = ViewRequest(kind=kind, scalar_field=handle if kind in (0, 1) else 0, vector_field=handle if kind == VIEW_VECTOR_FIELD else 0, consumer_stream=None)
        ptr = [c_void_p(t.data_ptr()) for t in outs] + [None] * (3 - len(outs))
        self._check(self.lib.stable_fluids_b200_read_view_async(self.ctx, byref(req), ptr[0], ptr[1], ptr[2], c_void_p(copy_stream.cuda_stream)), "read_view_async")

    # ------------------------------------------------------------- step --
    def step(self, n: int = 1):
        for _ in range(n):
            self._check(self.lib.stable_fluids_step_cuda(self.ctx), "step")

    def synchronize(self):
        self.stream.synchronize()
        self._keep.clear()

    # ---------------------------------------------------------- outputs --
    def raw_view(self, kind: int, handle: int = 0) -> View:
        req = ViewRequest(kind=kind, scalar_field=handle if kind in (0, 1) else 0, vector_field=handle if kind == VIEW_VECTOR_FIELD else 0, consumer_stream=c_void_p(self.stream.cuda_stream))
        v = View()
        self._check(self.lib.stable_fluids_get_view_cuda(self.ctx, byref(req), byref(v)), "get_view")
        return v

    def view(self, kind: int, handle: int = 0):
        """Zero-copy torch tensors on the library's memory (valid until the
        next step); a tuple of three for the vector layouts."""
        torch = self._torch
        v = self.raw_view(kind, handle)
        shape = (v.nz, v.ny, v.nx)
        ts = [torch.as_tensor(_DeviceArray(p, shape), device=self.device) for p in (v.data0, v.data1, v.data2) if p]
        return tuple(ts) if kind in (VIEW_FLOW_VELOCITY, VIEW_VECTOR_FIELD) else ts[0]

    def fetch(self, kind: int, handle: int = 0):
        """Host copies (numpy float32, shape (nz, ny, nx)) of a view."""
        torch = self._torch
        v = self.view(kind, handle)
        with torch.cuda.stream(self.stream):
            if isinstance(v, tuple):
                out = tuple(t.clone() for t in v)
            else:
                out = v.clone()
        self.stream.synchronize()
        if isinstance(out, tuple):
            return tuple(t.cpu().numpy() for t in out)
        return out.cpu().numpy()

    def stats(self) -> B200StepStats:
        s = B200StepStats()
        self._check(self.lib.stable_fluids_b200_get_step_stats(self.ctx, byref(s)), "get_step_stats")
        return s

    def info(self) -> B200StepInfo:
        i = B200StepInfo()
        self._check(self.lib.stable_fluids_b200_get_step_info(self.ctx, byref(i)), "get_step_info")
        return i

    def render_volume(self, kind: int, params, handle: int = 0, out=None):
        """Ray-marches the field of view kind `kind` (a single-array kind) into an
        RGBA float image (stable_fluids_b200_render_volume): a torch tensor
        (height, width, 4) on the simulation's device. The image is written on
        the simulation's stream; torch's current stream is made to wait for it."""
        torch = self._torch
        if out is None:
            with torch.cuda.stream(self.stream):
                out = torch.empty((params.height, params.width, 4), dtype=torch.float32, device=self.device)
        req = ViewRequest(kind=kind, scalar_field=handle if kind in (0, 1) else 0, vector_field=0, consumer_stream=c_void_p(self.stream.cuda_stream))
        self._check(self.lib.stable_fluids_b200_render_volume(self.ctx, byref(req), byref(params), c_void_p(out.data_ptr())), "render_volume")
        torch.cuda.current_stream(self.device).wait_stream(self.stream)
        return out

    def plume_scene_setup(self, density: int | None = None, force: int | None = None):
        """The reference viewer's plume inputs, generated on the device: density
        source and force y of the source sphere, force x and z zero
        (stable_fluids_b200_plume_scene_setup)."""
        d = self.scalar_handles[0] if density is None else density
        f = self.vector_handles[0] if force is None else force
        self._check(self.lib.stable_fluids_b200_plume_scene_setup(self.ctx, d, f), "plume_scene_setup")

    def plume_scene_forces(self, animation_step: int, force: int | None = None):
        """Force x and z of the viewer's plume for one animation step, written on
        the device into the force field (stable_fluids_b200_plume_scene_forces)."""
        f = self.vector_handles[0] if force is None else force
        self._check(self.lib.stable_fluids_b200_plume_scene_forces(self.ctx, f, int(animation_step)), "plume_scene_forces")

    def enqueue_stage(self, stage: int) -> int:
        """Enqueues one stage outside the step graph; returns its kernel count."""
        n = ctypes.c_int32(0)
        self._check(self.lib.stable_fluids_b200_enqueue_stage(self.ctx, stage, byref(n)), "enqueue_stage")
        return n.value

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.stable_fluids_destroy_context_cuda(self.ctx)
            self.ctx = None
        self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several Simulations stepped together (stable_fluids_b200_batch_*).

    mode: BATCH_GRAPHS (default: one graph of the simulations' step graphs)
    or BATCH_WORK_TABLE (one persistent launch per stage over L2-sized groups
    of simulations, groups on `chains` concurrent streams (0: 4); needs
    simulations with the same stage structure; the faster layout). autotune: time the sweep tile
    options per grid size at creation (work table), caching them in
    `tile_cache` (a JSON file) when given. After creation, `mode` is the
    layout in use, `groups` the number of L2-sized groups the work table runs
    one after another, and `z_chunks` the planes per thread block of each
    simulation's sweeps (work table)."""

    def __init__(self, simulations, mode: int | None = None, autotune: bool = False, tile_cache: str | os.PathLike | None = None, chains: int = 0):
        import torch

        from . import B200BatchOptions, BATCH_GRAPHS

        self.sims = list(simulations)
        if not self.sims:
            raise ValueError("empty batch")
        self.lib = self.sims[0].lib
        ctxs = (c_void_p * len(self.sims))(*[s.ctx for s in self.sims])
        h = c_void_p()
        opts = B200BatchOptions()
        opts.mode = BATCH_GRAPHS if mode is None else int(mode)
        opts.autotune = 1 if autotune else 0
        opts.chains = int(chains)
        self._cache = os.fsencode(str(tile_cache)) if tile_cache is not None else None
        opts.tile_cache = self._cache
        rc = self.lib.stable_fluids_b200_batch_create_ex(ctxs, len(self.sims), byref(opts), byref(h))
        if rc != RESULT_OK:
            raise StableFluidsError("stable_fluids_b200_batch_create_ex", rc)
        self.handle = h
        n, k, st = ctypes.c_uint32(0), ctypes.c_int32(0), c_void_p()
        self.lib.stable_fluids_b200_batch_info(h, byref(n), byref(k), byref(st))
        self.kernels_per_step = k.value
        m, g = ctypes.c_uint32(0), ctypes.c_uint32(0)
        zc = (ctypes.c_int32 * len(self.sims))()
        self.lib.stable_fluids_b200_batch_layout(h, byref(m), byref(g), zc, len(self.sims))
        self.mode = m.value
        self.groups = g.value
        self.z_chunks = list(zc)
        self.stream = torch.cuda.ExternalStream(st.value, device=self.sims[0].device)

    def step(self, n: int = 1):
        for _ in range(n):
            rc = self.lib.stable_fluids_b200_batch_step(self.handle)
            if rc != RESULT_OK:
                raise StableFluidsError("stable_fluids_b200_batch_step", rc)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.stable_fluids_b200_batch_destroy(self.handle)
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
