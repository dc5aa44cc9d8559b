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


def _bench_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("steps,warmup,chunk", [(20, 5, 50), (5000, 200, 50), (1, 3, 50), (3000, 3, 7),
                                                (123, 4, 10)])
def test_bench_stream_covers_every_consumer(steps, warmup, chunk):
    """The 1M workload's MF stream has a row for every step each part of
    bench.py reads: the timed runs, the kernel-timing copy, the per-step
    C-ABI run and the CPU baseline's sample (the driver's --steps 20
    --warmup 5 included)."""
    b = _bench_module()
    plan = b.stream_plan(steps, warmup, chunk)
    rows = plan["rows"]
    assert plan["main"] == warmup + 2 * steps
    assert plan["n_roof"] % chunk == 0 and plan["n_roof"] > 0
    assert plan["roofline"] == plan["n_fl"] + plan["n_roof"] + 2 * chunk
    assert plan["e2e"] == 20 + plan["n_e2e"]
    assert plan["cpu"] == b.CPU_WARMUP + b.CPU_STEPS
    for k in ("main", "roofline", "e2e", "cpu"):
        assert plan[k] <= rows, k


def test_cpu_baseline_rejects_a_short_stream(tmp_path):
    """A stream shorter than the CPU sample is refused before the harness
    runs (the failure the driver's first run met)."""
    b = _bench_module()
    import shutil
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_run")):
        pytest.skip("reference harness oracle/_ref not built")
    with pytest.raises(ValueError):
        b.cpu_reference(str(tmp_path / "none.state"), np.zeros((45, 1024), np.uint8), b.CPU_STEPS, 1,
                        warmup=b.CPU_WARMUP)
    del shutil


def test_bench_launches_ranks_itself_dry_run():
    """`bench.py --gpus 2 --dry-run` starts two processes itself (under
    torch.distributed.run, gloo), and rank 0 reports a world of 2."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run", "--steps", "5",
                        "--warmup", "3"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["ranks"] == 2 and len(set(d["pids"])) == 2


def test_reference_arm_prints_one_contract_line():
    """--impl reference prints one contract line, and its process never maps
    the product's CUDA library (the network is built by the oracle)."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '3', '--warmup', '3']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('MAPS_PRODUCT', 'libcbm_b200' in maps)")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MAPS_PRODUCT False" in r.stdout
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


@pytest.mark.parametrize("tau", [4.0, 10.0, 37.5, 100.0])
def test_mf_threshold_decay_constant_is_the_references(tmp_path, tau):
    """PoissonRegenCells' threshDecay = 1 - exp(-msPerTS / threshDecayTau)
    (CBM_TOOLS_LIB_DEV/src/poissonregencells.cpp:20) with float operands: in
    C++ that exp is the float overload, so the constant is 1.0f - expf(x).
    The expression is compiled here as C++ with the reference's header
    (<math.h>) and its result compared with the host generator's constant.
    At 4 ms a double exp rounded to float gives the same value; at the
    other time constants it does not."""
    import shutil
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "decay.cpp"
    src.write_text('#include <math.h>\n#include <stdio.h>\n#include <stdlib.h>\n'
                   'int main(int c, char **v) { float msPerTS = 1, threshDecayTau = strtof(v[1], 0);\n'
                   '  float threshDecay = 1 - exp(-msPerTS / threshDecayTau);\n'
                   '  printf("%.9e\\n", (double)threshDecay); return 0; }\n')
    exe = tmp_path / "decay"
    subprocess.run([gxx, "-O2", "-ffp-contract=off", str(src), "-o", str(exe)], check=True)
    ref = np.float32(float(subprocess.run([str(exe), repr(tau)], capture_output=True, text=True,
                                          check=True).stdout))
    got = networks.RegenPoissonMF(8, 1, thresh_decay_tau=tau).thresh_decay
    assert got == ref


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


@pytest.mark.parametrize("pre,post", [(40, 40), (48, 48)])
def test_raster_getters_count_completed_trials(tmp_path, pre, post):
    """A raster read back from a data file reports the raster's completed
    trials (curTrialN) as SpikeRasterBitArray::getNumTrials does.  With a
    160-step window, 4 updates fill each 5-row raster trial short of its
    last row: 2 trials x 4 updates = 8 rows, one completed trial.  With a
    176-step window (a multiple of 32 plus 16) it is 2 x 5 = 10 updates of 5
    rows: 2 trials."""
    from cerebellum_simulation_b200.trialdata import TrialsData, write_ec_trials_data
    proto = dict(preCS=pre, postCS=post, csOn=100, csOff=180, binSteps=16, numDataTrials=2)
    rec_len = pre + 80 + post
    bins = -(-rec_len // 16)
    cells = {"go": 8, "grInputGO": 8, "goInputGO": 8, "goOutSynScale": 8, "mf": 16, "sc": 4, "bc": 4, "pc": 2,
             "io": 1}
    rng = np.random.Generator(np.random.PCG64(1))
    td = {"psh": {n: rng.random((bins, c)).astype(np.float32) for n, c in cells.items()},
          "raster": {n: rng.integers(0, 2 ** 32, (2, rec_len // 32, c), dtype=np.uint32)
                     for n, c in (("go", 8), ("sc", 4), ("bc", 4), ("pc", 2), ("nc", 3), ("io", 1))}}
    path = str(tmp_path / "data")
    write_ec_trials_data(path, td, rng.integers(0, 9, (bins, 40)), rng.random((2, rec_len)), proto, 40)
    updates, rows = 2 * ((rec_len - 1) // 32), rec_len // 32
    assert updates // rows == ({160: 1, 176: 2}[rec_len])
    r = TrialsData.from_file(path).getRaster("go")
    assert r.getNumTrials() == updates // rows
    assert len(r.getCellSpikeTimes(0)) == updates // rows


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
