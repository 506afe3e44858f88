"""The allocation-free residual entry point against the library's own
residual measurement.

stable_fluids_b200_pressure_residual_noalloc() exists for callers that cannot
allocate device memory when they need the number (allocation-free frame
phases, fully pooled device memory, host callbacks); it keeps its scratch in
a fixed device array inside the library. This file is named so that pytest
collects it last: if it fails, a run stopped at the first failure has already
run every other test.
"""

import ctypes

import numpy as np
import pytest


def _residual_noalloc(sf, lib, sim, out):
    cfg = sim.config
    p = sim.raw_view(sf.VIEW_FLOW_PRESSURE).data0
    dv = sim.raw_view(sf.VIEW_FLOW_DIVERGENCE).data0
    rc = lib.stable_fluids_b200_pressure_residual_noalloc(p, dv, cfg.nx, cfg.ny, cfg.nz, cfg.cell_size, ctypes.byref(cfg.flow_boundary), out.data_ptr(), ctypes.c_void_p(sim.stream.cuda_stream))
    assert rc == sf.RESULT_OK
    sim.stream.synchronize()
    return out.cpu().numpy().copy()


@pytest.mark.gpu
@pytest.mark.parametrize("walls", ["stam", "benchmark"])
def test_noalloc_residual_matches_step_residual(walls, sf, lib, cuda):
    torch = cuda
    w = sf.scenes.stam_walls() if walls == "stam" else sf.scenes.benchmark_walls()
    scene = sf.scenes.plume("noalloc", (40, 32, 24), sources=[(20, 6, 12, 4.0, 10.0, 5.0)], velocity_seed=3, diffuse_iterations=4, pressure_iterations=10, walls=w)
    opts = sf.default_options(lib)
    opts.compute_residual = 1
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib, options=opts)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for call in range(2):  # two calls in a row, on different states
        sf.scenes.run(sim, scene, steps=2, start=2 * call)
        # the existing path: the projection stage measures the residual of
        # the context's current pressure and divergence into its scratch
        sim.enqueue_stage(sf.STAGE_PROJECTION)
        st = sim.stats()
        got = _residual_noalloc(sf, lib, sim, out)
        assert st.rel_residual > 0 and np.isfinite(got).all()
        np.testing.assert_allclose(got[0], st.rel_residual, rtol=1e-9)
        np.testing.assert_allclose(got[1], st.rhs_norm, rtol=1e-9)
    sim.close()


@pytest.mark.gpu
def test_noalloc_residual_rejects_grids_beyond_its_scratch(sf, lib, cuda):
    torch = cuda
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(1, dtype=torch.float32, device="cuda")
    walls = sf.scenes.stam_walls()[0]
    rc = lib.stable_fluids_b200_pressure_residual_noalloc(dummy.data_ptr(), dummy.data_ptr(), 2, 2, 4097, 0.1, ctypes.byref(walls), out.data_ptr(), None)
    assert rc == sf.RESULT_BACKEND_FAILURE


@pytest.mark.gpu
def test_noalloc_residual_rejects_invalid_arguments(sf, lib, cuda):
    """Every invalid argument is refused before any work is enqueued: null
    pointers, a non-positive or NaN cell size, an unknown face kind and an
    unpaired periodic face. A valid call with the same buffers succeeds."""
    torch = cuda
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    field = torch.zeros(4 * 4 * 4, dtype=torch.float32, device="cuda")
    sc = sf.scenes
    walls = sc.stam_walls()[0]
    unpaired = sc.flow_boundary([sf.FLOW_PERIODIC, sf.FLOW_FREE_SLIP_WALL] + [sf.FLOW_FREE_SLIP_WALL] * 4)
    unknown = sc.flow_boundary([7] + [sf.FLOW_FREE_SLIP_WALL] * 5)
    fn = lib.stable_fluids_b200_pressure_residual_noalloc
    p, q, o = field.data_ptr(), field.data_ptr(), out.data_ptr()
    bad = [
        (None, q, 4, 4, 4, 0.25, ctypes.byref(walls), o),
        (p, None, 4, 4, 4, 0.25, ctypes.byref(walls), o),
        (p, q, 4, 4, 4, 0.25, None, o),
        (p, q, 4, 4, 4, 0.25, ctypes.byref(walls), None),
        (p, q, 4, 4, 4, 0.0, ctypes.byref(walls), o),
        (p, q, 4, 4, 4, float("nan"), ctypes.byref(walls), o),
        (p, q, 0, 4, 4, 0.25, ctypes.byref(walls), o),
        (p, q, 4, 4, 4, 0.25, ctypes.byref(unknown), o),
        (p, q, 4, 4, 4, 0.25, ctypes.byref(unpaired), o),
    ]
    for args in bad:
        assert fn(*args, None) == sf.RESULT_BACKEND_FAILURE, args
    assert fn(p, q, 4, 4, 4, 0.25, ctypes.byref(walls), o, None) == sf.RESULT_OK
    torch.cuda.synchronize()
    assert out[0].item() == 0.0  # zero right-hand side: residual defined as 0
