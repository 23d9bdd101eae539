"""CPU checks of the C-ABI boundary: the library and header agree, the
library loads without a GPU, and host-side logic (problem set-up, params)
behaves."""
import ctypes
import os
import re

import numpy as np
import pytest

from css_b200 import _lib, params, problem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "css_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(css_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    if not os.path.exists(_lib.LIBPATH):
        pytest.skip("library not built")
    L = ctypes.CDLL(_lib.LIBPATH)
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_lib.EXPORTS) == sorted(n for n in names)


def test_params_struct_matches_header_field_count():
    src = open(os.path.join(ROOT, "include", "css_b200.h")).read()
    body = src[src.index("typedef struct css_params {"):src.index("} css_params;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    decl = re.findall(r"\b(int|double)\s+([^;]+);", body)
    count = sum(len(names.split(",")) for _, names in decl)
    assert count == len(params.CssParams._fields_)
    # same order and types
    flat = []
    for t, names in decl:
        for nm in names.split(","):
            flat.append((nm.strip(), t))
    for (nm, t), (fn, ft) in zip(flat, params.CssParams._fields_):
        assert nm == fn
        assert (t == "int") == (ft is ctypes.c_int)


def test_create_without_gpu_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    if not os.path.exists(_lib.LIBPATH):
        pytest.skip("library not built")
    from css_b200.context import Simulation
    p, prof, v0, dt, _ = problem.build((64, 64, 96), decomp=(2, 2, 3))
    with pytest.raises(_lib.CssError) as e:
        Simulation(p, prof)
    assert e.value.code in (3, 6)


def test_problem_setup_is_seeded_and_stratified():
    p, prof, v0, dt, info = problem.build("hydro-64x64x128")
    p2, prof2, v02, dt2, _ = problem.build("hydro-64x64x128")
    assert np.array_equal(v0, v02) and dt == dt2
    pr = prof.reshape(params.NPROF, p.nr)
    assert abs(np.log(pr[5][0] / pr[5][-1]) - 3.0) < 1e-12  # 3 density scale heights
    assert pr[1][0] == pytest.approx(0.70) and pr[1][-1] == pytest.approx(0.97)
    assert np.all(np.diff(pr[1]) > 0)
    # tanh stretching clusters points toward the top
    assert np.diff(pr[1])[-1] < np.diff(pr[1])[0]
    assert 1e-5 < dt < 1e-2
    _, _, v03, _, _ = problem.build("hydro-64x64x128", seed=7)
    assert not np.array_equal(v0, v03)
