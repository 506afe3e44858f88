"""Parity of libstable-fluids.so (through the C ABI) against the CPU oracle and
against the reference library itself, on the GPU.

Error measure: max |a - b| / max(|b|, FLOOR * max|b|) over every cell of
every output field (velocity x/y/z, pressure, divergence, |u|, each scalar).
"""

import numpy as np
import pytest

from tests.golden import cases as C

# The required bound against the reference library is 1e-5 max relative
# error (floor 1e-3 of the field scale). The RBGS scheme computes the
# reference's arithmetic in the same order, so it is held to bit equality.
REF_TOL, REF_FLOOR = 1e-5, 1e-3
# Against the FP32 CPU oracle (which is itself bit-equal to the reference):
# bit equality for RBGS; Jacobi has no reference counterpart and is held to
# 1e-5 against the oracle's Jacobi scheme.
ORACLE_TOL, ORACLE_FLOOR = 1e-5, 1e-3


def assert_bit_equal(a, b):
    diff = {k: int(np.sum(np.asarray(a[k], np.float32) != np.asarray(b[k], np.float32))) for k in b}
    assert not any(diff.values()), diff

CASES = {c.name: c for c in C.build_cases()}


def run_lib(sf, lib, case, steps=None, options=None):
    sim = sf.Simulation(case.config, case.scalars, case.vectors, lib=lib, options=options)
    case.drive(sim, steps)
    out = C.collect_outputs(sim, sf, case)
    sim.close()
    return out


def run_oracle(orc, case, steps=None, scheme=0, precision=32, **solver):
    o = orc.Oracle(case.config, case.scalars, case.vectors, precision=precision, scheme=scheme)
    if solver:
        o.set_solver(**solver)
    case.drive(o, steps)
    out = C.collect_oracle(o, orc, case)
    return out, o


def errors(a, b, floor):
    return {k: C.max_rel_err(a[k], b[k], floor) for k in b}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_rbgs_matches_reference_library(name, sf, lib, ref_lib, cuda):
    case = CASES[name]
    ours = run_lib(sf, lib, case)
    ref = run_lib(sf, ref_lib, case)
    err = errors(ours, ref, REF_FLOOR)
    assert max(err.values()) <= REF_TOL, err
    assert_bit_equal(ours, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_rbgs_matches_oracle(name, sf, lib, orc, cuda):
    case = CASES[name]
    ours = run_lib(sf, lib, case)
    ref, _ = run_oracle(orc, case)
    assert_bit_equal(ours, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_jacobi_matches_oracle(name, sf, lib, orc, cuda):
    case = CASES[name]
    opts = sf.default_options(lib)
    opts.scheme = sf.SCHEME_JACOBI
    ours = run_lib(sf, lib, case, options=opts)
    ref, _ = run_oracle(orc, case, scheme=orc.JACOBI)
    err = errors(ours, ref, ORACLE_FLOOR)
    assert max(err.values()) <= ORACLE_TOL, err


@pytest.mark.gpu
def test_config0_100_steps_matches_reference(sf, lib, ref_lib, cuda):
    """The 64^3 Stam-walls plume, 100 steps, against the reference library."""
    scene = sf.scenes.config0()
    outs = []
    for L in (lib, ref_lib):
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=L)
        sf.scenes.run(sim, scene)
        case = C.Case("config0", scene.config, scene.scalars, scene.vectors, scene.steps)
        outs.append(C.collect_outputs(sim, sf, case))
        sim.close()
    err = errors(outs[0], outs[1], REF_FLOOR)
    assert max(err.values()) <= REF_TOL, err
    assert_bit_equal(outs[0], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("warm", [False, True])
def test_residual_matches_oracle(warm, sf, lib, orc, cuda):
    case = CASES["walls_16x12x10"]
    opts = sf.default_options(lib)
    opts.compute_residual = 1
    opts.warm_start = sf.WARM_START_PREVIOUS if warm else sf.WARM_START_ZERO
    sim = sf.Simulation(case.config, case.scalars, case.vectors, lib=lib, options=opts)
    case.drive(sim)
    st = sim.stats()
    p = sim.fetch(sf.VIEW_FLOW_PRESSURE)
    sim.close()
    ref, o = run_oracle(orc, case, warm_previous=warm, compute_residual=True)
    ost = o.stats()
    assert st.pressure_iterations == case.config.pressure_iterations
    assert abs(st.rel_residual - ost["rel_residual"]) <= 1e-4 * ost["rel_residual"] + 1e-7, (st.rel_residual, ost)
    assert abs(st.rhs_norm - ost["rhs_norm"]) <= 1e-4 * ost["rhs_norm"]
    assert C.max_rel_err(p, ref["pressure"], ORACLE_FLOOR) <= ORACLE_TOL


@pytest.mark.gpu
def test_abi_error_paths(sf, lib, cuda):
    import ctypes

    case = CASES["walls_16x12x10"]
    sim = sf.Simulation(case.config, case.scalars, case.vectors, lib=lib)
    ctx = sim.ctx
    # bad handles (upstream :695, :704, :713, :762)
    assert lib.stable_fluids_update_scalar_field_cuda(ctx, 0, None) == sf.RESULT_BACKEND_FAILURE
    assert lib.stable_fluids_update_scalar_field_cuda(ctx, 2, None) == sf.RESULT_BACKEND_FAILURE
    assert lib.stable_fluids_update_scalar_field_source_cuda(ctx, 7, None) == sf.RESULT_BACKEND_FAILURE
    assert lib.stable_fluids_update_vector_field_cuda(ctx, 0, None, None, None) == sf.RESULT_BACKEND_FAILURE
    req = sf.ViewRequest(kind=99)
    v = sf.View()
    assert lib.stable_fluids_get_view_cuda(ctx, ctypes.byref(req), ctypes.byref(v)) == sf.RESULT_BACKEND_FAILURE
    req = sf.ViewRequest(kind=sf.VIEW_SCALAR_FIELD_DATA, scalar_field=5)
    assert lib.stable_fluids_get_view_cuda(ctx, ctypes.byref(req), ctypes.byref(v)) == sf.RESULT_BACKEND_FAILURE
    assert lib.stable_fluids_step_cuda(None) == sf.RESULT_BACKEND_FAILURE
    assert lib.stable_fluids_get_view_cuda(None, ctypes.byref(req), ctypes.byref(v)) == sf.RESULT_BACKEND_FAILURE
    # null pointer = zero fill (upstream :697)
    assert lib.stable_fluids_update_scalar_field_cuda(ctx, 1, None) == sf.RESULT_OK
    assert not sim.fetch(sf.VIEW_SCALAR_FIELD_DATA, 1).any()
    # views are dense, x-fastest (upstream :732-742)
    v = sim.raw_view(sf.VIEW_FLOW_VELOCITY)
    assert v.layout == sf.VIEW_LAYOUT_F32_3D_SOA3 and v.row_stride_bytes == 4 * v.nx and v.slice_stride_bytes == 4 * v.nx * v.ny
    assert sim.raw_view(sf.VIEW_FLOW_PRESSURE).layout == sf.VIEW_LAYOUT_F32_3D
    sim.close()
    assert lib.stable_fluids_destroy_context_cuda(None) == sf.RESULT_OK


@pytest.mark.gpu
@pytest.mark.parametrize("walls", ["stam", "benchmark"])
def test_diverged_velocity_stays_in_bounds(walls, sf, lib, cuda):
    """A force of +-inf or NaN (a diverged simulation) makes back-traced
    positions infinite or NaN; the advection gathers must still read inside
    the fields (the step completes and the views are readable)."""
    sc = sf.scenes
    scene = _tiled_scene(sf, (16, 12, 10), sc.stam_walls() if walls == "stam" else sc.benchmark_walls(), steps=2)
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib)
    n = 16 * 12 * 10
    fx, fy, fz = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32)
    fx[5], fy[700], fz[1200] = np.inf, -np.inf, np.nan
    fx[1500] = 3.0e38
    sim.set_vector(sim.vector_handles[0], fx, fy, fz)
    sim.step(2)
    sim.synchronize()
    vel = sim.fetch(sf.VIEW_FLOW_VELOCITY)
    assert all(v.shape == (10, 12, 16) for v in vel)
    sim.close()


def _create_rc(sf, lib, cfg, scalars=(), vectors=()):
    import ctypes

    sa = (sf.ScalarFieldDesc * max(1, len(scalars)))(*scalars)
    va = (sf.VectorFieldDesc * max(1, len(vectors)))(*vectors)
    desc = sf.ContextCreateDesc(config=cfg, stream=None, scalar_fields=ctypes.cast(sa, ctypes.POINTER(sf.ScalarFieldDesc)), scalar_field_count=len(scalars), vector_fields=ctypes.cast(va, ctypes.POINTER(sf.VectorFieldDesc)), vector_field_count=len(vectors))
    ctx = ctypes.c_void_p()
    rc = lib.stable_fluids_create_context_cuda(ctypes.byref(desc), ctypes.byref(ctx), None, 0, None, 0)
    if rc == sf.RESULT_OK:
        lib.stable_fluids_destroy_context_cuda(ctx)
    return rc


@pytest.mark.gpu
def test_create_validation(sf, lib, cuda):
    sc = sf.scenes
    good = sc.make_config((8, 8, 8), 0.125, 0.1, 1e-4, 2, 2, sc.stam_walls()[0])
    assert _create_rc(sf, lib, good) == sf.RESULT_OK
    # unpaired periodic face (upstream :519)
    bad = sc.make_config((8, 8, 8), 0.125, 0.1, 1e-4, 2, 2, sc.flow_boundary([sf.FLOW_PERIODIC, sf.FLOW_FREE_SLIP_WALL] + [sf.FLOW_FREE_SLIP_WALL] * 4))
    assert _create_rc(sf, lib, bad) == sf.RESULT_BACKEND_FAILURE
    # unknown kind (upstream :517)
    bad = sc.make_config((8, 8, 8), 0.125, 0.1, 1e-4, 2, 2, sc.flow_boundary([7] + [sf.FLOW_FREE_SLIP_WALL] * 5))
    assert _create_rc(sf, lib, bad) == sf.RESULT_BACKEND_FAILURE
    # scalar periodic unpaired (upstream :524)
    s = sf.ScalarFieldDesc(0, 0, 0, sc.scalar_boundary([sf.SCALAR_PERIODIC] + [sf.SCALAR_ZERO_FLUX] * 5))
    assert _create_rc(sf, lib, good, [s]) == sf.RESULT_BACKEND_FAILURE
    # stricter than upstream: empty grid, non-positive cell size, negative iterations
    assert _create_rc(sf, lib, sc.make_config((0, 8, 8), 0.125, 0.1, 1e-4, 2, 2, sc.stam_walls()[0])) == sf.RESULT_BACKEND_FAILURE
    assert _create_rc(sf, lib, sc.make_config((8, 8, 8), 0.0, 0.1, 1e-4, 2, 2, sc.stam_walls()[0])) == sf.RESULT_BACKEND_FAILURE
    assert _create_rc(sf, lib, sc.make_config((8, 8, 8), 0.125, 0.1, 1e-4, -1, 2, sc.stam_walls()[0])) == sf.RESULT_BACKEND_FAILURE


@pytest.mark.gpu
def test_out_of_memory_paths(sf, lib, cuda, monkeypatch):
    sc = sf.scenes
    # host-side fault injection: the allocation reports failure
    monkeypatch.setenv("STABLE_FLUIDS_B200_INJECT_ALLOC_FAILURE", "1")
    good = sc.make_config((8, 8, 8), 0.125, 0.1, 1e-4, 2, 2, sc.stam_walls()[0])
    assert _create_rc(sf, lib, good) == sf.RESULT_OUT_OF_MEMORY
    monkeypatch.delenv("STABLE_FLUIDS_B200_INJECT_ALLOC_FAILURE")
    # a real allocation larger than the device: 4096^3 cells x 15 fields
    huge = sc.make_config((4096, 4096, 4096), 1.0 / 4096, 0.1, 1e-4, 2, 2, sc.stam_walls()[0])
    assert _create_rc(sf, lib, huge) == sf.RESULT_OUT_OF_MEMORY
    assert _create_rc(sf, lib, good) == sf.RESULT_OK  # the device is still usable


@pytest.mark.gpu
def test_views_and_consumer_stream(sf, lib, cuda):
    torch = cuda
    case = CASES["benchmark_walls_16x12x16"]
    sim = sf.Simulation(case.config, case.scalars, case.vectors, lib=lib)
    case.drive(sim)
    consumer = torch.cuda.Stream()
    import ctypes

    req = sf.ViewRequest(kind=sf.VIEW_SCALAR_FIELD_SOURCE, scalar_field=2, consumer_stream=ctypes.c_void_p(consumer.cuda_stream))
    v = sf.View()
    assert lib.stable_fluids_get_view_cuda(sim.ctx, ctypes.byref(req), ctypes.byref(v)) == sf.RESULT_OK
    t = torch.as_tensor(sf.simulation._DeviceArray(v.data0, case.shape), device="cuda")
    with torch.cuda.stream(consumer):
        got = t.clone()
    consumer.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), case.sources[2])
    fx, fy, fz = sim.fetch(sf.VIEW_VECTOR_FIELD, 2)
    np.testing.assert_array_equal(fx, case.forces[2][0])
    sim.close()


def _tiled_scene(sf, n, walls, steps=3):
    """Grids large enough for several xy tiles and z chunks of the blocked
    stencil (TMA path when nx % 4 == 0, cp.async path otherwise)."""
    nx, ny, nz = n
    return sf.scenes.plume("tiled", n, dt=0.1, viscosity=1e-4, diffusion=1e-5, diffuse_iterations=5, pressure_iterations=7, sources=[(nx / 2, 6, nz / 2, 5.0, 10.0, 6.0), (nx / 4, 5, nz / 3, 4.0, 8.0, 3.0)], walls=walls, velocity_seed=2, steps=steps)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["walls_200x60x40", "benchmark_192x56x36", "walls_odd_181x47x29"])
def test_tiled_grids_match_reference_library(kind, sf, lib, ref_lib, cuda):
    if kind == "walls_200x60x40":
        scene = _tiled_scene(sf, (200, 60, 40), sf.scenes.stam_walls())
    elif kind == "benchmark_192x56x36":
        scene = _tiled_scene(sf, (192, 56, 36), sf.scenes.benchmark_walls())
    else:
        scene = _tiled_scene(sf, (181, 47, 29), sf.scenes.stam_walls())
    outs = []
    for L in (lib, ref_lib):
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=L)
        sf.scenes.run(sim, scene)
        case = C.Case(kind, scene.config, scene.scalars, scene.vectors, scene.steps)
        outs.append(C.collect_outputs(sim, sf, case))
        sim.close()
    err = errors(outs[0], outs[1], REF_FLOOR)
    assert max(err.values()) <= REF_TOL, err
    assert_bit_equal(outs[0], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_blocked_rbgs_matches_reference_library(name, sf, lib, ref_lib, cuda):
    """The temporally blocked passes (two RBGS iterations per HBM pass)
    reproduce the reference bit for bit."""
    case = CASES[name]
    opts = sf.default_options(lib)
    opts.iterations_per_pass = 2
    ours = run_lib(sf, lib, case, options=opts)
    ref = run_lib(sf, ref_lib, case)
    assert_bit_equal(ours, ref)


@pytest.mark.gpu
def test_blocked_rbgs_tiled_grid_matches_reference_library(sf, lib, ref_lib, cuda):
    scene = _tiled_scene(sf, (200, 60, 40), sf.scenes.benchmark_walls())
    outs = []
    for L, o in ((lib, 2), (ref_lib, None)):
        opts = None
        if o is not None:
            opts = sf.default_options(lib)
            opts.iterations_per_pass = o
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=L, options=opts)
        sf.scenes.run(sim, scene)
        outs.append(C.collect_outputs(sim, sf, C.Case("t", scene.config, scene.scalars, scene.vectors, scene.steps)))
        sim.close()
    assert_bit_equal(outs[0], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["walls_16x12x10", "benchmark_walls_16x12x16", "mixed_odd_17x9x13"])
@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("warm", [False, True])
def test_residual_driven_solve_matches_oracle(name, scheme, warm, sf, lib, orc, cuda):
    """Pressure iterated inside the step graph (WHILE node) until the FP64
    relative residual <= 1e-3: same iteration counts, residuals and fields as
    the oracle's loop."""
    case = CASES[name]
    tol, interval, cap = 1e-3, 4, 2000
    opts = sf.default_options(lib)
    opts.scheme = scheme
    opts.residual_tolerance = tol
    opts.residual_check_interval = interval
    opts.max_pressure_iterations = cap
    opts.warm_start = sf.WARM_START_PREVIOUS if warm else sf.WARM_START_ZERO
    sim = sf.Simulation(case.config, case.scalars, case.vectors, lib=lib, options=opts)
    o = orc.Oracle(case.config, case.scalars, case.vectors, precision=32, scheme=scheme)
    o.set_solver(tolerance=tol, max_iterations=cap, check_interval=interval, warm_previous=warm)
    for k in range(case.steps):
        case.drive(sim, steps=1, start=k)
        case.drive(o, steps=1, start=k)
        st = sim.stats()
        ost = o.stats()
        info = (k, st.pressure_iterations, st.rel_residual, st.hit_cap, ost)
        assert st.pressure_iterations == ost["iterations"], info
        assert st.hit_cap == ost["hit_cap"], info
        assert st.rel_residual <= tol or st.hit_cap == 1
        assert abs(st.rel_residual - ost["rel_residual"]) <= 1e-6 * ost["rel_residual"] + 1e-12
    ours = C.collect_outputs(sim, sf, case)
    ref = C.collect_oracle(o, orc, case)
    sim.close()
    err = errors(ours, ref, ORACLE_FLOOR)
    assert max(err.values()) <= ORACLE_TOL, err


@pytest.mark.gpu
def test_residual_driven_solve_stops_at_cap(sf, lib, cuda):
    case = CASES["walls_16x12x10"]
    opts = sf.default_options(lib)
    opts.residual_tolerance = 1e-9
    opts.residual_check_interval = 4
    opts.max_pressure_iterations = 10  # rounded up to 12
    sim = sf.Simulation(case.config, case.scalars, case.vectors, lib=lib, options=opts)
    case.drive(sim, steps=1)
    st = sim.stats()
    sim.close()
    assert st.hit_cap == 1 and st.pressure_iterations == 12 and st.rel_residual > 1e-9


def _wave_scene(sf, kind):
    """Grids whose rows suit the z-wavefront passes (nx = 128 or 256), with
    several tiles and z chunks, partial last tiles and every boundary kind."""
    sc = sf.scenes
    if kind == "stam_128x44x37":
        return _tiled_scene(sf, (128, 44, 37), sc.stam_walls())
    if kind == "benchmark_256x30x22":
        return _tiled_scene(sf, (256, 30, 22), sc.benchmark_walls())
    if kind == "periodic_y_128x24x40":
        flow = sc.flow_boundary([sf.FLOW_NO_SLIP_WALL, sf.FLOW_FREE_SLIP_WALL, sf.FLOW_PERIODIC, sf.FLOW_PERIODIC, sf.FLOW_OUTFLOW, sf.FLOW_FREE_SLIP_WALL], pressures=[0, 0, 0, 0, 0.25, 0])
        sbc = sc.scalar_boundary([sf.SCALAR_FIXED_VALUE, sf.SCALAR_ZERO_FLUX, sf.SCALAR_PERIODIC, sf.SCALAR_PERIODIC, sf.SCALAR_ZERO_FLUX, sf.SCALAR_FIXED_VALUE], values=[0.5, 0, 0, 0, 0, 1.5])
        return _tiled_scene(sf, (128, 24, 40), (flow, sbc))
    if kind == "periodic_xz_256x12x10":
        flow = sc.flow_boundary([sf.FLOW_PERIODIC, sf.FLOW_PERIODIC, sf.FLOW_NO_SLIP_WALL, sf.FLOW_OUTFLOW, sf.FLOW_PERIODIC, sf.FLOW_PERIODIC], velocities=[(0, 0, 0)] * 2 + [(0.3, 0, -0.2), (0, 0, 0)] + [(0, 0, 0)] * 2)
        sbc = sc.scalar_boundary([sf.SCALAR_PERIODIC, sf.SCALAR_PERIODIC, sf.SCALAR_ZERO_FLUX, sf.SCALAR_FIXED_VALUE, sf.SCALAR_PERIODIC, sf.SCALAR_PERIODIC])
        return _tiled_scene(sf, (256, 12, 10), (flow, sbc))
    raise KeyError(kind)


WAVE_KINDS = ["stam_128x44x37", "benchmark_256x30x22", "periodic_y_128x24x40", "periodic_xz_256x12x10"]


def _run_scene(sf, lib, scene, options=None):
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib, options=options)
    sf.scenes.run(sim, scene)
    out = C.collect_outputs(sim, sf, C.Case(scene.name, scene.config, scene.scalars, scene.vectors, scene.steps))
    sim.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("kind", WAVE_KINDS)
def test_wave_jacobi_matches_single_sweeps(kind, sf, lib, cuda):
    """K Jacobi sweeps per HBM pass (the z-wavefront kernel, asked for with
    2, 3 or 4 iterations per pass) give the same bits as one sweep per launch
    (the default, 0, and 1), across tile and z-chunk seams, partial tiles,
    every face kind and periodic axes."""
    scene = _wave_scene(sf, kind)
    outs = {}
    for per_pass in (1, 0, 2, 3, 4):
        opts = sf.default_options(lib)
        opts.scheme = sf.SCHEME_JACOBI
        opts.iterations_per_pass = per_pass
        outs[per_pass] = _run_scene(sf, lib, scene, opts)
    for per_pass in (0, 2, 3, 4):
        assert_bit_equal(outs[per_pass], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", WAVE_KINDS)
def test_wave_rbgs_matches_reference_library(kind, sf, lib, ref_lib, cuda):
    """Red-black iterations in z-wavefront passes (2 and 4 iterations per
    pass asked for) are bit-equal to the reference library, and so is one
    launch per colour (the default)."""
    scene = _wave_scene(sf, kind)
    ref = _run_scene(sf, ref_lib, scene)
    for per_pass in (0, 2, 4):
        opts = sf.default_options(lib)
        opts.iterations_per_pass = per_pass
        assert_bit_equal(_run_scene(sf, lib, scene, opts), ref)


def _rb_split_scene(sf, kind):
    """Grids at the edges of the split-layout red-black solve: colour rows of
    one float4 and of 64 and 128, a row length it leaves to the colour
    launches (12), odd y and z sizes, and periodic axes down to two planes."""
    sc = sf.scenes
    periodic = (sc.flow_boundary([sf.FLOW_PERIODIC] * 6), sc.scalar_boundary([sf.SCALAR_PERIODIC] * 6))
    grids = {
        "narrow_8x9x7": ((8, 9, 7), sc.stam_walls()),
        "narrow_12x31x6": ((12, 31, 6), sc.benchmark_walls()),
        "wide_512x11x9": ((512, 11, 9), sc.stam_walls()),
        "wide_1024x7x6": ((1024, 7, 6), sc.benchmark_walls()),
        "periodic_16x6x2": ((16, 6, 2), periodic),
        "periodic_64x10x12": ((64, 10, 12), periodic),
    }
    n, walls = grids[kind]
    return _tiled_scene(sf, n, walls)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["narrow_8x9x7", "narrow_12x31x6", "wide_512x11x9", "wide_1024x7x6", "periodic_16x6x2", "periodic_64x10x12"])
def test_rbgs_split_matches_colour_launches(kind, sf, lib, ref_lib, cuda):
    """Red-black solves in the split layout (the default for FP32 fields)
    give the bits of the colour launches on the interleaved field
    (iterations_per_pass = 1) and of the reference library."""
    scene = _rb_split_scene(sf, kind)
    outs = {}
    for per_pass in (0, 1):
        opts = sf.default_options(lib)
        opts.iterations_per_pass = per_pass
        outs[per_pass] = _run_scene(sf, lib, scene, opts)
    assert_bit_equal(outs[0], outs[1])
    assert_bit_equal(outs[0], _run_scene(sf, ref_lib, scene))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["narrow_8x9x7", "wide_512x11x9", "periodic_64x10x12"])
def test_rbgs_split_bf16_matches_colour_launches(kind, sf, lib, cuda):
    """BF16 storage: the split-layout diffusion solves give the bits of the
    BF16 colour launches (FP32 arithmetic, one rounding to BF16 per update)."""
    scene = _rb_split_scene(sf, kind)
    outs = {}
    for per_pass in (0, 1):
        opts = sf.default_options(lib)
        opts.storage = sf.STORAGE_BF16
        opts.iterations_per_pass = per_pass
        outs[per_pass] = _run_scene(sf, lib, scene, opts)
    assert_bit_equal(outs[0], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["stam_128x44x37", "periodic_xz_256x12x10"])
def test_wave_jacobi_matches_oracle(kind, sf, lib, orc, cuda):
    """The Jacobi scheme (numerator times the rounded reciprocal) against the
    FP32 oracle's Jacobi, on grids the wavefront kernel takes."""
    scene = _wave_scene(sf, kind)
    opts = sf.default_options(lib)
    opts.scheme = sf.SCHEME_JACOBI
    opts.iterations_per_pass = 3
    ours = _run_scene(sf, lib, scene, opts)
    case = C.Case(scene.name, scene.config, scene.scalars, scene.vectors, scene.steps)
    o = orc.Oracle(scene.config, scene.scalars, scene.vectors, precision=32, scheme=orc.JACOBI)
    sf.scenes.run(o, scene)
    ref = C.collect_oracle(o, orc, case)
    err = errors(ours, ref, ORACLE_FLOOR)
    assert max(err.values()) <= ORACLE_TOL, err


def _batch_vs_single(sf, lib, scenes, options=None, **batch_kw):
    """Steps each scene alone, then all of them as one batch; returns the
    batch layout and, per simulation, (batch outputs, single outputs, batch
    stats, single stats)."""
    single, single_stats = [], []
    for sc in scenes:
        sim = sf.Simulation(sc.config, sc.scalars, sc.vectors, lib=lib, options=options)
        sf.scenes.run(sim, sc)
        single.append(C.collect_outputs(sim, sf, C.Case(sc.name, sc.config, sc.scalars, sc.vectors, sc.steps)))
        single_stats.append(sim.stats())
        sim.close()
    sims = [sf.Simulation(sc.config, sc.scalars, sc.vectors, lib=lib, options=options) for sc in scenes]
    for sim, sc in zip(sims, scenes):
        sf.scenes.apply_inputs(sim, sc, 0)
    out = []
    with sf.Batch(sims, **batch_kw) as batch:
        batch.step(scenes[0].steps)
        info = {"mode": batch.mode, "kernels": batch.kernels_per_step, "z_chunks": batch.z_chunks}
    for sim, sc, ref, ref_st in zip(sims, scenes, single, single_stats):
        out.append((C.collect_outputs(sim, sf, C.Case(sc.name, sc.config, sc.scalars, sc.vectors, sc.steps)), ref, sim.stats(), ref_st))
        sim.close()
    return info, out


@pytest.mark.gpu
def test_batch_graphs_match_single_contexts(sf, lib, cuda):
    """GRAPHS layout: the contexts' step graphs as children of one graph give
    the same bits as stepping each context on its own."""
    scenes = sf.scenes.batch_scenes(count=4, seed=7, steps=3)
    kernels = []
    for sc in scenes:
        sim = sf.Simulation(sc.config, sc.scalars, sc.vectors, lib=lib)
        kernels.append(sim.info().kernels_per_step)
        sim.close()
    info, out = _batch_vs_single(sf, lib, scenes, mode=sf.BATCH_GRAPHS)
    assert info["mode"] == sf.BATCH_GRAPHS and info["kernels"] == sum(kernels)
    for got, ref, _, _ in out:
        assert_bit_equal(got, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme,chains", [(0, 1), (1, 1), (0, 3)])
def test_batch_work_table_matches_single_contexts(scheme, chains, sf, lib, cuda):
    """WORK_TABLE layout: one persistent launch per stage over all
    simulations (uneven sizes) gives the same bits as stepping each context on
    its own, for both schemes (Jacobi with the previous-pressure start and the
    per-simulation FP64 residual) and with the groups on concurrent streams."""
    scenes = sf.scenes.batch_scenes(count=5, seed=11, steps=3)
    opts = sf.default_options(lib)
    opts.scheme = scheme
    if scheme == 1:
        opts.warm_start = sf.WARM_START_PREVIOUS
        opts.compute_residual = 1
    info, out = _batch_vs_single(sf, lib, scenes, options=opts, mode=sf.BATCH_WORK_TABLE, chains=chains)
    assert info["mode"] == sf.BATCH_WORK_TABLE
    assert all(z > 0 for z in info["z_chunks"])
    for got, ref, st, ref_st in out:
        assert_bit_equal(got, ref)
        if scheme == 1:
            assert st.pressure_iterations == ref_st.pressure_iterations
            assert st.rel_residual == pytest.approx(ref_st.rel_residual, rel=1e-9, abs=1e-30)


@pytest.mark.gpu
def test_batch_work_table_autotune_and_cache(sf, lib, cuda, tmp_path):
    """The tile autotuner picks a z chunk per grid size, writes the JSON
    cache, and a second batch reads the same choices back; results stay
    bit-equal to single contexts."""
    import json

    scenes = sf.scenes.batch_scenes(count=4, seed=3, steps=2)
    cache = tmp_path / "tiles.json"
    info, out = _batch_vs_single(sf, lib, scenes, mode=sf.BATCH_WORK_TABLE, autotune=True, tile_cache=cache)
    for got, ref, _, _ in out:
        assert_bit_equal(got, ref)
    table = json.loads(cache.read_text())
    sizes = {sc.config.nx for sc in scenes}
    assert len(table) == len(sizes)
    for key, zc in table.items():
        n = int(key.rsplit("|", 1)[1].split("x")[2])
        assert 1 <= zc <= n
    sims = [sf.Simulation(sc.config, sc.scalars, sc.vectors, lib=lib) for sc in scenes]
    with sf.Batch(sims, mode=sf.BATCH_WORK_TABLE, autotune=True, tile_cache=cache) as batch:
        assert batch.z_chunks == info["z_chunks"]
    for sim in sims:
        sim.close()


@pytest.mark.gpu
def test_batch_work_table_needs_common_stages(sf, lib, cuda):
    """Contexts whose stage structure differs (here BF16 storage in one of
    them) batch as GRAPHS and are refused for WORK_TABLE."""
    scenes = sf.scenes.batch_scenes(count=2, seed=5, steps=1)
    bf = sf.default_options(lib)
    bf.storage = sf.STORAGE_BF16
    sims = [sf.Simulation(scenes[0].config, scenes[0].scalars, scenes[0].vectors, lib=lib), sf.Simulation(scenes[1].config, scenes[1].scalars, scenes[1].vectors, lib=lib, options=bf)]
    with sf.Batch(sims) as batch:
        assert batch.mode == sf.BATCH_GRAPHS
    with pytest.raises(sf.StableFluidsError):
        sf.Batch(sims, mode=sf.BATCH_WORK_TABLE)
    for sim in sims:
        sim.close()


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [0, 1])
def test_bf16_storage_against_fp64_oracle(scheme, sf, lib, orc, cuda):
    """BF16 storage of velocity and density (FP32 arithmetic, FP32 pressure):
    the error against the FP64 oracle stays within a few BF16 roundings
    (2^-8 relative) per field, close to the FP32 library's own error."""
    scene = sf.scenes.config0(steps=20)
    outs = {}
    for storage in (sf.STORAGE_FP32, sf.STORAGE_BF16):
        opts = sf.default_options(lib)
        opts.scheme = scheme
        opts.storage = storage
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib, options=opts)
        sf.scenes.run(sim, scene)
        outs[storage] = {"density": sim.fetch(sf.VIEW_SCALAR_FIELD_DATA, sim.scalar_handles[0]), "velocity": np.stack(sim.fetch(sf.VIEW_FLOW_VELOCITY)), "pressure": sim.fetch(sf.VIEW_FLOW_PRESSURE)}
        sim.close()
    o = orc.Oracle(scene.config, scene.scalars, scene.vectors, precision=64, scheme=scheme)
    sf.scenes.run(o, scene)
    ref = {"density": o.get(orc.SCALAR, 1), "velocity": np.stack(o.velocity()), "pressure": o.get(orc.PRESSURE)}
    errs = {k: (rel_l2(outs[sf.STORAGE_FP32][k], ref[k]), rel_l2(outs[sf.STORAGE_BF16][k], ref[k])) for k in ref}
    print("relative L2 error vs FP64 (FP32 storage, BF16 storage):", errs)
    for k, (e32, e16) in errs.items():
        assert e16 <= 2e-2, (k, errs)
        assert e32 <= 1e-4, (k, errs)


@pytest.mark.gpu
def test_batch_shares_one_network(sf, lib, cuda):
    """Learned-start contexts of different sizes attached to one warm-start
    network step together in a GRAPHS batch (each predicts with its own
    activation buffers) and give the same bits as stepping each alone with
    that network; destroying a context after the network is safe."""
    scenes = [sf.scenes.plume(f"shared-net-{n}", (n, n, n), sources=[(n / 2, 5, n / 2, 3.0, 10.0, 5.0)], diffuse_iterations=2, pressure_iterations=24, steps=3) for n in (16, 16, 24)]
    opts = sf.default_options(lib)
    opts.scheme = sf.SCHEME_JACOBI
    opts.warm_start = sf.WARM_START_LEARNED
    opts.compute_residual = 1
    net = sf.WarmStartNetwork(seed=0, lib=lib)
    single = []
    for sc in scenes:
        sim = sf.Simulation(sc.config, sc.scalars, sc.vectors, lib=lib, options=opts)
        net.attach(sim)
        sf.scenes.run(sim, sc)
        single.append((C.collect_outputs(sim, sf, C.Case(sc.name, sc.config, sc.scalars, sc.vectors, sc.steps)), sim.stats().rel_residual))
        sim.close()
    sims = [sf.Simulation(sc.config, sc.scalars, sc.vectors, lib=lib, options=opts) for sc in scenes]
    for sim, sc in zip(sims, scenes):
        net.attach(sim)
        sf.scenes.apply_inputs(sim, sc, 0)
    with sf.Batch(sims, mode=sf.BATCH_GRAPHS) as batch:
        for k in range(scenes[0].steps):
            if k == 1:
                for sim, sc in zip(sims, scenes):
                    sf.scenes.apply_inputs(sim, sc, 1)
            batch.step(1)
    for sim, sc, (ref, ref_res) in zip(sims, scenes, single):
        assert_bit_equal(C.collect_outputs(sim, sf, C.Case(sc.name, sc.config, sc.scalars, sc.vectors, sc.steps)), ref)
        assert sim.stats().rel_residual == pytest.approx(ref_res, rel=1e-9)  # FP64 sums by atomics: order varies
    net.close()
    for sim in sims:  # after the network: nothing of it is touched
        sim.close()
