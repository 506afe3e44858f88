"""The staged input upload and the asynchronous view read-back
(stable_fluids_b200_stage_vector_field, stable_fluids_b200_read_view_async)
give the same steps and the same data as update_vector_field and the views."""

import numpy as np
import pytest


def _scene(sf):
    return sf.scenes.plume("async_io", (32, 24, 20), sources=[(16, 6, 10, 3.0, 10.0, 5.0)], velocity_seed=1, diffuse_iterations=6, pressure_iterations=12, steps=4)


@pytest.mark.gpu
def test_staged_upload_and_async_readback_match(sf, lib, cuda):
    import torch

    scene = _scene(sf)
    n = 32 * 24 * 20
    rng = np.random.default_rng(3)
    forces = [[rng.standard_normal(n).astype(np.float32) for _ in range(3)] for _ in range(scene.steps)]
    forces[2][1] = None  # a null component zero-fills
    # reference: update_vector_field, then the views
    ref = []
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib)
    sf.scenes.apply_inputs(sim, scene, 0)
    for f in forces:
        sim.set_vector(sim.vector_handles[0], *f)
        sim.step(1)
        ref.append((sim.fetch(sf.VIEW_SCALAR_FIELD_DATA, sim.scalar_handles[0]), sim.fetch(sf.VIEW_FLOW_VELOCITY)))
    sim.close()
    # staged upload on a copy stream, asynchronous read-back
    copy = torch.cuda.Stream()
    pinned = [[None if a is None else torch.from_numpy(a).pin_memory() for a in f] for f in forces]
    rho = [torch.empty(n, dtype=torch.float32).pin_memory() for _ in forces]
    vel = [[torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(3)] for _ in forces]
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib)
    sf.scenes.apply_inputs(sim, scene, 0)
    for k, f in enumerate(pinned):
        sim.stage_vector(sim.vector_handles[0], *f, copy)
        sim.step(1)
        sim.read_view_async(sf.VIEW_SCALAR_FIELD_DATA, [rho[k]], copy, handle=sim.scalar_handles[0])
        sim.read_view_async(sf.VIEW_FLOW_VELOCITY, vel[k], copy)
    copy.synchronize()
    sim.synchronize()
    sim.close()
    for k, (r_rho, r_vel) in enumerate(ref):
        assert np.array_equal(rho[k].numpy().view(np.uint32), r_rho.reshape(-1).view(np.uint32)), k
        for a, b in zip(vel[k], r_vel):
            assert np.array_equal(a.numpy().view(np.uint32), b.reshape(-1).view(np.uint32)), k


@pytest.mark.gpu
def test_async_io_rejects_bad_arguments(sf, lib, cuda):
    import ctypes
    import torch

    scene = _scene(sf)
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib)
    copy = torch.cuda.Stream()
    cs = ctypes.c_void_p(copy.cuda_stream)
    assert lib.stable_fluids_b200_stage_vector_field(sim.ctx, 0, None, None, None, cs) == sf.RESULT_BACKEND_FAILURE  # handle 0
    assert lib.stable_fluids_b200_stage_vector_field(sim.ctx, 1, None, None, None, None) == sf.RESULT_BACKEND_FAILURE  # no copy stream
    req = sf.ViewRequest(kind=sf.VIEW_FLOW_VELOCITY)
    out = torch.empty(32 * 24 * 20, dtype=torch.float32).pin_memory()
    # a three-array view with one destination
    assert lib.stable_fluids_b200_read_view_async(sim.ctx, ctypes.byref(req), ctypes.c_void_p(out.data_ptr()), None, None, cs) == sf.RESULT_BACKEND_FAILURE
    sim.close()
