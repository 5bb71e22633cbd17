"""The integral files (cl_write_integrals, coulombo.cpp:213-262) byte for byte against the
oracle's restatement of the reference's serial writer, on one and on many host threads."""
import os

import numpy as np
import pytest

import coulombo_lattice_b200 as cl
from oracle import host as H


@pytest.mark.parametrize("holes,electrons,pattern", [(2, 2, "****"), (6, 6, "eeee,hhhh,ehhe,eheh"),
                                                     (3, 5, "ijji,1*2*"), (10, 10, "****")])
@pytest.mark.parametrize("threads", [1, 0])
def test_files_match_the_serial_writer(tmp_path, holes, electrons, pattern, threads):
    n = holes + electrons
    specs = H.enumerate_integrals(H.Pattern(pattern, holes), n)
    rng = np.random.default_rng(n * 31 + holes)
    # values spanning signs and magnitudes, some exactly representable
    vals = (rng.standard_normal(len(specs)) * 10.0 ** rng.integers(-12, 2, len(specs))
            + 1j * rng.standard_normal(len(specs)) * 10.0 ** rng.integers(-12, 2, len(specs)))
    vals[:3] = [0.0, -1.5 + 0.25j, 1e-20 - 1e-20j]
    out = str(tmp_path) + os.sep
    cl.write_integrals(out, holes, electrons, specs, vals, threads=threads)
    want = H.format_outputs(specs, list(vals), holes, electrons)
    assert sorted(f for f in os.listdir(tmp_path)) == sorted(k + ".txt" for k in want)
    for core, text in want.items():
        with open(os.path.join(str(tmp_path), core + ".txt")) as fh:
            assert fh.read() == text


def test_rejects_out_of_range_specs(tmp_path):
    with pytest.raises(cl.CoulomboError, match="out of range"):
        cl.write_integrals(str(tmp_path) + os.sep, 1, 1, [(1, 2, 3, 1)], [1.0])
