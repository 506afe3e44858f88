"""CPU checks of the drop-in boundary: exported symbols and the binary layout
of every ABI struct and enum (no GPU, no compute calls)."""

import ctypes
import os
import pathlib
import re
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
INCLUDE = ROOT / "include"
REFERENCE = pathlib.Path(os.environ.get("STABLE_FLUIDS_REFERENCE", "/root/reference"))


def declared_functions():
    names = []
    for h in sorted(INCLUDE.glob("*.h")):
        names += re.findall(r"STABLE_FLUIDS_API\s+StableFluidsResult\s+(\w+)\s*\(", h.read_text())
    return names


def test_header_declares_the_upstream_entry_points(sf):
    names = declared_functions()
    for s in sf.ABI_SYMBOLS + sf.B200_SYMBOLS:
        assert s in names


def test_library_exports_every_declared_symbol(sf):
    lib_path = sf.LIB_PATH
    assert lib_path.exists(), "build the library first (__graft_entry__.build())"
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], check=True, capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    # only the ABI is exported (no CUDA runtime or C++ internals)
    extra = [s for s in exported if not s.startswith("stable_fluids_")]
    assert not extra, extra[:10]
    lib = sf.load_library()  # loads with ctypes; no CUDA call is made
    assert lib._sf_extended


STRUCTS = ["StableFluidsFlowBoundaryFaceDesc", "StableFluidsFlowBoundaryConfig", "StableFluidsScalarBoundaryFaceDesc", "StableFluidsScalarBoundaryConfig", "StableFluidsSimulationConfig", "StableFluidsScalarFieldDesc",
           "StableFluidsVectorFieldDesc", "StableFluidsContextCreateDesc", "StableFluidsViewRequest", "StableFluidsView"]
ENUMS = ["STABLE_FLUIDS_RESULT_OK", "STABLE_FLUIDS_RESULT_OUT_OF_MEMORY", "STABLE_FLUIDS_RESULT_BACKEND_FAILURE", "STABLE_FLUIDS_FLOW_BOUNDARY_NO_SLIP_WALL", "STABLE_FLUIDS_FLOW_BOUNDARY_FREE_SLIP_WALL",
         "STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW", "STABLE_FLUIDS_FLOW_BOUNDARY_PERIODIC", "STABLE_FLUIDS_SCALAR_BOUNDARY_FIXED_VALUE", "STABLE_FLUIDS_SCALAR_BOUNDARY_ZERO_FLUX",
         "STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC", "STABLE_FLUIDS_VECTOR_FIELD_FORCE", "STABLE_FLUIDS_VIEW_SCALAR_FIELD_DATA", "STABLE_FLUIDS_VIEW_SCALAR_FIELD_SOURCE", "STABLE_FLUIDS_VIEW_VECTOR_FIELD",
         "STABLE_FLUIDS_VIEW_FLOW_VELOCITY", "STABLE_FLUIDS_VIEW_FLOW_VELOCITY_MAGNITUDE", "STABLE_FLUIDS_VIEW_FLOW_PRESSURE", "STABLE_FLUIDS_VIEW_FLOW_DIVERGENCE",
         "STABLE_FLUIDS_VIEW_LAYOUT_F32_3D", "STABLE_FLUIDS_VIEW_LAYOUT_F32_3D_SOA3"]


def ctypes_struct(sf, cname):
    return {
        "StableFluidsFlowBoundaryFaceDesc": sf.FlowFace, "StableFluidsFlowBoundaryConfig": sf.FlowBoundary, "StableFluidsScalarBoundaryFaceDesc": sf.ScalarFace,
        "StableFluidsScalarBoundaryConfig": sf.ScalarBoundary, "StableFluidsSimulationConfig": sf.SimulationConfig, "StableFluidsScalarFieldDesc": sf.ScalarFieldDesc,
        "StableFluidsVectorFieldDesc": sf.VectorFieldDesc, "StableFluidsContextCreateDesc": sf.ContextCreateDesc, "StableFluidsViewRequest": sf.ViewRequest, "StableFluidsView": sf.View,
    }[cname]


def layout_from_compiler(sf, include_dir, tmp_path):
    """sizeof/offsetof of every struct field and every enum value, as a C
    compiler sees `stable-fluids-3d.h` in include_dir."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "stable-fluids-3d.h"', "int main(void) {"]
    for cname in STRUCTS:
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in ctypes_struct(sf, cname)._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    for e in ENUMS:
        lines.append(f'printf("{e} %d\\n", (int){e});')
    lines += ["return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", str(include_dir), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return dict(line.rsplit(" ", 1) for line in out.splitlines())


def test_ctypes_mirror_matches_our_header(sf, tmp_path):
    got = layout_from_compiler(sf, INCLUDE, tmp_path)
    for cname in STRUCTS:
        cls = ctypes_struct(sf, cname)
        assert int(got[f"{cname} sizeof"]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)


@pytest.mark.skipif(not (REFERENCE / "stable-fluids-3d.h").exists(), reason="reference header not present")
def test_layout_identical_to_reference_header(sf, tmp_path):
    (tmp_path / "ours").mkdir()
    (tmp_path / "ref").mkdir()
    ours = layout_from_compiler(sf, INCLUDE, tmp_path / "ours")
    theirs = layout_from_compiler(sf, REFERENCE, tmp_path / "ref")
    assert ours == theirs


def test_enum_values(sf):
    assert (sf.RESULT_OK, sf.RESULT_OUT_OF_MEMORY, sf.RESULT_BACKEND_FAILURE) == (0, 1, 2)
    assert (sf.FLOW_NO_SLIP_WALL, sf.FLOW_FREE_SLIP_WALL, sf.FLOW_OUTFLOW, sf.FLOW_PERIODIC) == (0, 1, 2, 3)
    assert (sf.SCALAR_FIXED_VALUE, sf.SCALAR_ZERO_FLUX, sf.SCALAR_PERIODIC) == (0, 1, 2)
    assert sf.VIEW_FLOW_DIVERGENCE == 6 and sf.VIEW_LAYOUT_F32_3D_SOA3 == 1


EXT_STRUCTS = {"StableFluidsB200Options": "B200Options", "StableFluidsB200StepStats": "B200StepStats", "StableFluidsB200StepInfo": "B200StepInfo",
               "StableFluidsB200BatchOptions": "B200BatchOptions", "StableFluidsB200VolumeRender": "B200VolumeRender"}


def test_ctypes_mirror_matches_extension_header(sf, tmp_path):
    """The binding's copies of the extension structs (stable-fluids-b200.h)
    have the compiler's sizes and field offsets."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "stable-fluids-b200.h"', "int main(void) {"]
    for cname, pyname in EXT_STRUCTS.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in getattr(sf, pyname)._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "probe_ext.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe_ext"
    subprocess.run(["gcc", "-std=c11", "-I", str(INCLUDE), str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines())
    for cname, pyname in EXT_STRUCTS.items():
        cls = getattr(sf, pyname)
        assert int(got[f"{cname} sizeof"]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)
