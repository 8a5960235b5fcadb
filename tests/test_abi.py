"""The C-ABI library loads and exports every symbol declared in include/clgpu.h
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from cuclarabel_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "clgpu.h")).read()
    return sorted(set(re.findall(r"\b(clgpu_[A-Za-z_]+)\s*\(", src)))


def test_library_exports_all_declared_symbols():
    L = _lib.load()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(names) == sorted(_lib.EXPORTED)


def test_default_settings_match_reference_defaults():
    L = _lib.load()
    s = _lib.ClgpuSettings()
    assert L.clgpu_default_settings(ctypes.byref(s)) == 0
    # src/settings.jl:70-148
    assert s.max_iter == 200 and s.max_step_fraction == 0.99
    assert s.tol_gap_abs == 1e-8 and s.tol_feas == 1e-8 and s.tol_ktratio == 1e-6
    assert s.static_regularization_constant == 1e-8
    assert s.iterative_refinement_max_iter == 10 and s.soc_threshold == 5


def test_create_rejects_bad_input_without_gpu_work():
    from cuclarabel_b200 import Settings
    import numpy as np
    import scipy.sparse as sp
    from cuclarabel_b200.api import _prep_problem
    import pytest
    with pytest.raises(ValueError):
        _prep_problem(sp.eye(2), np.zeros(2), sp.eye(3, 2), np.zeros(3), [])
    with pytest.raises(ValueError):
        Settings(direct_solve_method="qdldl").to_c()


def test_host_objects_hold_no_compiler_traps():
    """gcc turns undefined behaviour it can prove (a division by a constant
    zero, a null dereference on some path) into a trap instruction; the
    library's own host objects must hold none."""
    import shutil
    import subprocess
    import pytest
    build = os.path.join(os.path.dirname(_lib.LIB_PATH), "_build")
    objdump = shutil.which("objdump")
    if not objdump or not os.path.isdir(build):
        pytest.skip("objdump or the object directory is missing")
    bad = []
    for name in sorted(os.listdir(build)):
        if not name.endswith(".o"):
            continue
        out = subprocess.run([objdump, "-d", "--no-show-raw-insn", "-C",
                              os.path.join(build, name)],
                             capture_output=True, text=True).stdout
        fn = None
        for line in out.splitlines():
            m = re.match(r"^[0-9a-f]+ <(.*)>:$", line)
            if m:
                fn = m.group(1)
            elif "\tud2" in line:
                bad.append((name, fn))
    assert not bad, bad
