"""The C-ABI library loads and exports every symbol include/fwgpu.h declares."""
import os
import re
import subprocess

import pytest

from conftest import REPO, has_gpu


def header_functions():
    txt = open(os.path.join(REPO, "include", "fwgpu.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(fwgpu_\w+)\(", txt, flags=re.M)))


def test_header_declares_entry_points():
    fns = header_functions()
    assert "fwgpu_hddm_solve" in fns and "fwgpu_solve_dom_1st" in fns
    assert len(fns) >= 20


def test_library_exports_every_declared_symbol():
    from adventure_fullwave_b200 import _lib

    lib_path = _lib.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(fwgpu_\w+)", out))
    missing = [f for f in header_functions() if f not in exported]
    assert not missing, missing
    lib = _lib.load()
    for f in header_functions():
        assert getattr(lib, f) is not None


def test_binding_covers_header():
    from adventure_fullwave_b200 import _lib

    assert sorted(_lib.SIGNATURES) == header_functions()


def test_abi_version():
    from adventure_fullwave_b200 import _lib

    txt = open(os.path.join(REPO, "include", "fwgpu.h")).read()
    declared = int(re.search(r"^#define FWGPU_ABI_VERSION (\d+)", txt, flags=re.M).group(1))
    assert declared == 4  # 4: the correction-Jo entry points (fwgpu_cojo_*)
    assert _lib.load().fwgpu_abi_version() == declared


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    from adventure_fullwave_b200 import _lib, hddm, meshgen

    m = meshgen.make_model("tiny", n=4, npml=1, nleaves=4)
    with pytest.raises(_lib.FwgpuError) as e:
        hddm.HddmSolver(m)
    assert e.value.code == _lib.ERR_CUDA
