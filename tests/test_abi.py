"""The C-ABI library loads and exports every entry point declared in include/*.h; GPU entry
points fail cleanly (status code + message) when no GPU is present."""
import ctypes
import glob
import os
import re

import pytest

import coulombo_lattice_b200 as cl
from conftest import ROOT, has_gpu


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(cl_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    names = declared_symbols()
    assert len(names) >= 17
    L = ctypes.CDLL(cl.LIB_PATH)
    for n in names:
        assert hasattr(L, n), n


def test_python_mirror_binds_every_symbol():
    bound = {s[0] for s in cl.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_last_error_is_thread_local_and_cleared():
    L = cl.lib()
    assert L.cl_round_up_235(10, 0) == -1
    assert b"c must be" in L.cl_last_error()
    assert L.cl_round_up_235(10, 1) == 10
    assert L.cl_last_error() == b""


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_create_without_gpu_reports_error():
    with pytest.raises(cl.CoulomboError) as e:
        cl.CoulombCalculator((4, 4, 4))
    assert e.value.kind == "cuda" and "no CUDA device" in str(e.value)


def test_create_argument_checks():
    for dims, msg in [((7, 4, 4), "not a product of 2, 3 and 5"), ((0, 4, 4), "must be positive")]:
        with pytest.raises(cl.CoulomboError, match=msg):
            cl.CoulombCalculator(dims)
    with pytest.raises(cl.CoulomboError, match="step lengths"):
        cl.CoulombCalculator((4, 4, 4), step=(1, 0, 1))
