"""ctypes binding of the CPU oracle (sf_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker. The product never imports it.

`Oracle` mirrors the subset of `Simulation` the scene driver uses
(set_scalar_source, set_vector, set_scalar, step, fetch) so one driver feeds
identical inputs to the library under test and to the oracle.
"""

from __future__ import annotations

import ctypes
import pathlib
import subprocess
from ctypes import POINTER, byref, c_double, c_int, c_uint32, c_void_p

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libsf_oracle.so"
REF_LIB_PATH = HERE / "_ref" / "libstable-fluids-ref.so"

# field kinds of sfo_get_field / sfo_set_field
SCALAR, SOURCE, VECTOR, VELOCITY, MAGNITUDE, PRESSURE, DIVERGENCE, SCALAR_TEMP, VELOCITY_TEMP = range(9)
RBGS, JACOBI = 0, 1

_lib = None


def build():
    subprocess.run(["make", "-C", str(HERE), "_build/libsf_oracle.so"], check=True, capture_output=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.sfo_create.argtypes = [c_void_p, c_int, c_int, POINTER(c_void_p)]
    lib.sfo_create.restype = c_int
    lib.sfo_destroy.argtypes = [c_void_p]
    lib.sfo_set_solver.argtypes = [c_void_p, c_double, c_int, c_int, c_int, c_int]
    lib.sfo_set_sum_order.argtypes = [c_int]
    lib.sfo_set_threads.argtypes = [c_int]
    lib.sfo_set_threads.restype = c_int
    lib.sfo_set_field.argtypes = [c_void_p, c_int, c_uint32, c_int, c_void_p]
    lib.sfo_set_field.restype = c_int
    lib.sfo_get_field.argtypes = [c_void_p, c_int, c_uint32, c_int, c_void_p]
    lib.sfo_get_field.restype = c_int
    lib.sfo_step.argtypes = [c_void_p, c_int]
    lib.sfo_get_stats.argtypes = [c_void_p, POINTER(c_double), POINTER(c_double), POINTER(c_int), POINTER(c_int)]
    lib.sfo_rel_residual.argtypes = [c_void_p, POINTER(c_double)]
    lib.sfo_rel_residual.restype = c_double
    _lib = lib
    return lib


def set_threads(n: int) -> int:
    return load().sfo_set_threads(n)


def set_sum_order(order: int):
    load().sfo_set_sum_order(order)


class Oracle:
    def __init__(self, config, scalar_fields=(), vector_fields=(), *, precision=64, scheme=RBGS):
        sf = _package()
        self.lib = load()
        self.shape = (config.nz, config.ny, config.nx)
        self.cells = config.nx * config.ny * config.nz
        self._scalars = (sf.ScalarFieldDesc * max(1, len(scalar_fields)))(*scalar_fields)
        self._vectors = (sf.VectorFieldDesc * max(1, len(vector_fields)))(*vector_fields)
        desc = sf.ContextCreateDesc(config=config, stream=None, scalar_fields=ctypes.cast(self._scalars, POINTER(sf.ScalarFieldDesc)), scalar_field_count=len(scalar_fields), vector_fields=ctypes.cast(self._vectors, POINTER(sf.VectorFieldDesc)), vector_field_count=len(vector_fields))
        self._desc = desc
        h = c_void_p()
        rc = self.lib.sfo_create(ctypes.addressof(desc), precision, scheme, byref(h))
        if rc != 0:
            raise RuntimeError(f"sfo_create failed ({rc})")
        self.h = h

    def set_solver(self, tolerance=0.0, max_iterations=0, check_interval=1, warm_previous=False, compute_residual=False):
        self.lib.sfo_set_solver(self.h, tolerance, max_iterations, check_interval, int(warm_previous), int(compute_residual))

    def _set(self, kind, handle, comp, values):
        ptr = None
        if values is not None:
            a = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
            assert a.size == self.cells
            ptr = a.ctypes.data
        rc = self.lib.sfo_set_field(self.h, kind, handle, comp, ptr)
        if rc != 0:
            raise RuntimeError(f"sfo_set_field({kind}) failed ({rc})")

    def set_scalar(self, handle, values):
        self._set(SCALAR, handle, 0, values)

    def set_scalar_source(self, handle, values):
        self._set(SOURCE, handle, 0, values)

    def set_vector(self, handle, x, y, z):
        for k, v in enumerate((x, y, z)):
            self._set(VECTOR, handle, k, v)

    def set_velocity(self, x, y, z):
        for k, v in enumerate((x, y, z)):
            self._set(VELOCITY, 0, k, v)

    def set_pressure(self, p):
        self._set(PRESSURE, 0, 0, p)

    def step(self, n=1):
        self.lib.sfo_step(self.h, n)

    def get(self, kind, handle=0, comp=0):
        out = np.empty(self.cells, np.float64)
        rc = self.lib.sfo_get_field(self.h, kind, handle, comp, out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"sfo_get_field({kind}) failed ({rc})")
        return out.reshape(self.shape)

    def velocity(self):
        return tuple(self.get(VELOCITY, 0, k) for k in range(3))

    def stats(self):
        rr, bn, it, cap = c_double(), c_double(), c_int(), c_int()
        self.lib.sfo_get_stats(self.h, byref(rr), byref(bn), byref(it), byref(cap))
        return {"rel_residual": rr.value, "rhs_norm": bn.value, "iterations": it.value, "hit_cap": cap.value}

    def rel_residual(self):
        bn = c_double()
        return self.lib.sfo_rel_residual(self.h, byref(bn))

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _package():
    import importlib
    import sys

    root = str(HERE.parent)
    if root not in sys.path:
        sys.path.insert(0, root)
    return importlib.import_module("stable-fluids_b200")
