"""A C++ driver written against the reference's class names
(include/cbm_core.hpp) steps a network on the GPU and saves the same state
as the Python binding driven with the same inputs."""
import subprocess

import numpy as np
import pytest

import cbmtest

pytestmark = pytest.mark.gpu


def facade_mf(steps, num_mf=1024):
    # the spike pattern tests/cpp/facade_check.cpp feeds at step t
    i = np.arange(num_mf, dtype=np.uint64)
    out = np.empty((steps, num_mf), dtype=np.uint8)
    for t in range(steps):
        out[t] = ((i * np.uint64(2654435761) + np.uint64((t * 40503) & 0xFFFFFFFF)) % np.uint64(97)) < 3
    return out


def test_cpp_facade_steps_like_the_python_binding(tmp_path):
    import cerebellum_simulation_b200 as cbm
    exe = cbmtest.build_facade_check(str(tmp_path))
    p = cbmtest.golden_state("ref16k", str(tmp_path))
    out_cpp = str(tmp_path / "cpp.state")
    txt = subprocess.run([exe, p, out_cpp], check=True, capture_output=True, text=True).stdout
    assert "steps 50" in txt
    st = cbm.CBMState(p)
    sim = cbm.CBMSimCore(st, [7], device=0)
    cbmtest.product_run(sim, facade_mf(50), record=False)
    out_py = str(tmp_path / "py.state")
    sim.writeToState(out_py)
    assert open(out_cpp, "rb").read() == open(out_py, "rb").read()
