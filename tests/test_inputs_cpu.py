"""Host-side inputs and the benchmark's reference arm, without a GPU.

* The state-variable MF coding of the dense configuration: each variable's
  fibres blend their relaxed and excited rates by a Gaussian of the distance
  between the variable's value and the fibre's preferred value
  (StateVariable::gaussMFAct, Matthew_Sim_CBM/includes/statevariable.hpp:108-129).
* The regenerating Poisson fibres are a deterministic function of the seed.
* `bench.py --impl reference` prints one JSON line that carries the fields
  the benchmark contract asks for (or its `unavailable` line).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from cerebellum_simulation_b200 import networks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_state_variable_rates_follow_the_gaussian_tuning():
    c = networks.StateVariableMF(1024, seed=4)
    per = 1024 // 4
    for t in (1, 250, 777):
        r = c.rates(t)
        x = c.values(t)
        assert np.all(r >= c.relaxed - 1e-5) and np.all(r <= 40.0 + 1e-4)
        for v in range(4):
            share = slice(v * per, (v + 1) * per)
            a = (r[share] - c.relaxed[share]) / (c.excited[share] - c.relaxed[share])
            # the blend weight falls with the distance to the preferred value
            d = np.abs(c.mean[share] - x[v])
            order = np.argsort(d)
            assert np.all(np.diff(a[order]) <= 1e-5)
            want = np.exp(-(d * d) / (2 * c.variance * c.variance))
            assert np.allclose(a, want, atol=1e-5)


def test_config3_stream_is_deterministic():
    a = networks.config3_mf_stream(1024, 300, seed=2)
    b = networks.config3_mf_stream(1024, 300, seed=2)
    c = networks.config3_mf_stream(1024, 300, seed=3)
    assert a.dtype == np.uint8 and a.shape == (300, 1024)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    rate_hz = a.mean() * 1000.0
    assert 2.0 < rate_hz < 40.0


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "3",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["warmup"] == 3
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1


def test_random_mf_population_follows_the_reference_rules():
    """MFPopulation.random: the category counts and rate ranges of the
    reference's ECMFPopulation random constructor (ecmfpopulation.cpp:67-190)."""
    p = networks.MFPopulation.random(1024, 3, 0.05, 0.03, 0.1, 1, 2, 30, 60, 110, 10, 5, 40, 80, 150)
    bg, t, ph = p.bg, p.cs_tonic, p.cs_phasic
    tonic = (t != bg) & (t == ph)
    phasic = (ph != bg) & (t == bg)
    context = (bg >= 30) & (t == bg) & (ph == bg)
    assert tonic.sum() == int(np.float32(0.05) * np.float32(1024)) == 51
    assert phasic.sum() == 30 and context.sum() == 102
    assert np.all((t[tonic] >= 60) & (t[tonic] < 80)) and np.all((ph[phasic] >= 110) & (ph[phasic] < 150))
    assert np.all((bg[tonic | phasic] >= 2) & (bg[tonic | phasic] < 5))
    plain = ~(tonic | phasic | context)
    assert np.all((bg[plain] >= 1) & (bg[plain] < 10))
    q = networks.MFPopulation.random(1024, 3, 0.05, 0.03, 0.1, 1, 2, 30, 60, 110, 10, 5, 40, 80, 150)
    assert np.array_equal(q.rates(), p.rates())


def test_mf_population_file_round_trip_and_truncation(tmp_path):
    p = networks.MFPopulation.random(256, 1, 0.05, 0.05, 0.1, 1, 2, 30, 60, 110, 10, 5, 40, 80, 150)
    path = str(tmp_path / "pop")
    p.write(path)
    q = networks.MFPopulation.read(path)
    assert np.array_equal(p.rates(), q.rates())
    data = open(path, "rb").read()
    assert len(data) == 4 + 3 * 256 * 4
    with open(path, "wb") as f:
        f.write(data[:-4])
    with pytest.raises(ValueError):
        networks.MFPopulation.read(path)


def test_eyelid_out_smoothing_rule():
    """EyelidOut::updateData: the first three values as they are, then the
    mean of the three previous recorded values and the new one."""
    import cerebellum_simulation_b200 as cbm
    raw = np.arange(1, 9, dtype=np.float32)[None, :]
    out = cbm.eyelid_out(raw)
    want = list(raw[0, :3])
    for t in range(3, 8):
        want.append(np.float32((np.float32(want[t - 3] + want[t - 2]) + want[t - 1] + raw[0, t]) / 4))
    assert np.array_equal(out[0], np.array(want, np.float32))


def test_trial_data_file_reader_rejects_truncation(tmp_path):
    from cerebellum_simulation_b200.trialdata import read_ec_trials_data, write_ec_trials_data
    proto = dict(preCS=40, postCS=40, csOn=100, csOff=180, binSteps=10, numDataTrials=2)
    rec_len, cells = 160, {"go": 8, "grInputGO": 8, "goInputGO": 8, "goOutSynScale": 8, "mf": 16, "sc": 4,
                           "bc": 4, "pc": 2, "io": 1}
    rng = np.random.Generator(np.random.PCG64(0))
    td = {"psh": {n: rng.random((16, c)).astype(np.float32) for n, c in cells.items()},
          "raster": {n: rng.integers(0, 2 ** 32, (2, rec_len // 32, c), dtype=np.uint32)
                     for n, c in (("go", 8), ("sc", 4), ("bc", 4), ("pc", 2), ("nc", 3), ("io", 1))}}
    path = str(tmp_path / "data")
    write_ec_trials_data(path, td, rng.integers(0, 9, (16, 40)), rng.random((2, rec_len)), proto, 40)
    buf = open(path, "rb").read()
    back = read_ec_trials_data(buf)
    assert back["end"] == len(buf) and back["header"]["msTotal"] == rec_len
    for n, h in td["psh"].items():
        assert np.array_equal(back["psh"][n], h)
    for n, r in td["raster"].items():
        assert np.array_equal(back["raster"][n], r)
    assert back["psh"]["gr"].shape == (16, 4)
    with pytest.raises(ValueError):
        read_ec_trials_data(buf[: len(buf) // 2])
