"""Pins the CPU oracle to the reference.

The oracle (oracle/cbm_oracle.c) restates the reference's calcActivity; here
it must reproduce, bit for bit, the trace records and final state of the
reference's own host code:
  - against golden digests recorded from oracle/_ref/ref_run (always run);
  - against oracle/_ref/ref_run live, where the harness is built;
  - with the reference's GR-sharded multi-GPU host path (2 and 4 fake GPUs),
    which must equal its single-GPU result.
"""
import os

import numpy as np
import pytest

import cbmtest
from cbmtest import Oracle

EVENTS16K = {
    5: [("plast", 0, -0.01, 0.005)],
    700: [("errdrive", 0, 1.0)],
    1000: [("errdrive", 0, 0.6)],
    1200: [("plastreset", 0)],
    1300: [("grgoinc", 0.01)],
    1400: [("grgoincreset",)],
}


def test_oracle_matches_reference_golden_16k(tmp_path):
    gold = cbmtest.load_json("ref16k_digests.json")
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    o = Oracle(st, seeds=[7])
    mf = cbmtest.counter_mf(1024, gold["steps"], 11)
    tr = o.run(mf, EVENTS16K)
    assert tr.shape[1] == gold["record_bytes"]
    got = [cbmtest.sha(r) for r in tr]
    bad = [i for i, (a, b) in enumerate(zip(got, gold["records"])) if a != b]
    assert not bad, f"first differing step {bad[0] + 1}"
    fin = str(tmp_path / "final.state")
    o.save(fin)
    with open(fin, "rb") as f:
        assert cbmtest.sha(np.frombuffer(f.read(), np.uint8)) == gold["final_state"]


def test_oracle_matches_reference_golden_config1(tmp_path):
    from cerebellum_simulation_b200 import networks
    gold = cbmtest.load_json("config1_digests.json")
    net = networks.config1_network(seed=0)
    p = str(tmp_path / "c1.state")
    net.writeState(p)
    with open(p, "rb") as f:
        assert cbmtest.sha(np.frombuffer(f.read(), np.uint8)) == gold["initial_state"], \
            "config-1 generator is not deterministic"
    o = Oracle(p, seeds=[7])
    mf = networks.uniform_mf_stream(1024, gold["steps"], seed=0)
    tr = o.run(mf)
    got = [cbmtest.sha(r) for r in tr]
    bad = [i for i, (a, b) in enumerate(zip(got, gold["records"])) if a != b]
    assert not bad, f"first differing step {bad[0] + 1}"


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
@pytest.mark.parametrize("mf_seed,zone_seed", [(3, 99), (4, 12345)])
def test_oracle_matches_reference_live(tmp_path, mf_seed, zone_seed):
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    mf = cbmtest.counter_mf(1024, 800, mf_seed, rate_hi=0.1)
    ev = {3: [("plast", 0, -0.02, 0.01)], 400: [("errdrive", 0, 1.0)], 401: [("errdrive", 0, 0.2)]}
    fin_ref = str(tmp_path / "ref_final.state")
    ref = cbmtest.ref_run(st, mf, [zone_seed], ev, final_path=fin_ref).reshape(800, -1)
    o = Oracle(st, seeds=[zone_seed])
    tr = o.run(mf, ev)
    assert cbmtest.first_difference(ref, tr, o.num) is None
    fin = str(tmp_path / "oracle_final.state")
    o.save(fin)
    assert open(fin, "rb").read() == open(fin_ref, "rb").read()


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
@pytest.mark.parametrize("gpus", [2, 4])
def test_reference_sharded_path_equals_single(tmp_path, gpus):
    """The reference splits GR across GPUs and sums GR->GO counts on the
    host (innet.cpp:177, 835-838); with the fake runtime reporting several
    devices it must give the single-device result, which the oracle pins."""
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    mf = cbmtest.counter_mf(1024, 300, 5)
    single = cbmtest.ref_run(st, mf, [7], None)
    sharded = cbmtest.ref_run(st, mf, [7], None, num_gpus=gpus)
    assert np.array_equal(single, sharded)


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
@pytest.mark.parametrize("window", [dict(), dict(preCS=56, postCS=60), dict(mfThreshDecayTau=10.0),
                                    dict(mfThreshDecayTau=37.5)])
def test_oracle_protocol_matches_reference_driver(tmp_path, window):
    """The oracle's eyelid driver (MF generation, US, plasticity window,
    eyelid integrator, records) against the reference's PoissonRegenCells,
    EyelidIntegrator and ECTrialsData driven in the order of
    ECManagementDelay, over 3 short trials of the reference's 16K network.
    The second window is 256 steps long: 7 raster updates a trial against 8
    rows a raster trial, so the reference's raster trials drift across the
    protocol's trials, and the oracle must drift the same way.  The last two
    change the MF threshold recovery time constant: at 10 and 37.5 ms the
    float expf of poissonregencells.cpp:20 and a double exp rounded to float
    give different constants (at 4 ms they agree)."""
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol(**window)
    o = Oracle(st, seeds=[7])
    rates = cbmtest.protocol_rates(o.num["MF"], seed=1)
    steps = 3 * proto["trialSteps"]
    tr_o, nc, pc, eye, td = o.run_protocol(proto, rates, steps, trial_data=True)
    tr_r, rec_r = cbmtest.ref_run_protocol(st, proto, rates, steps, [7])
    assert tr_r.size == tr_o.size
    assert cbmtest.same_values(tr_r, tr_o.ravel()).all()
    r = cbmtest.split_ref_records(rec_r, o.num, proto)
    assert cbmtest.same_values(r["eye"], eye).all()
    assert np.array_equal(r["nc"], nc) and np.array_equal(r["pc"], pc)
    # the driver's smoothed eyelid record (EyelidOut) from the raw trace
    import cerebellum_simulation_b200 as cbm
    smooth = cbm.eyelid_out(eye.reshape(proto["numDataTrials"], -1))
    assert cbmtest.same_values(r["eyelid_out"].ravel(), smooth.ravel()).all()
    # the GR histogram rule the device follows, restated from the oracle's
    # trace, equals the reference's PeriStimHistFloat; the driver's own "gr"
    # histogram covers the first numGR / 10 cells
    gr_o = cbmtest.gr_psh_from_trace(tr_o, proto, o.num["GR"])
    assert gr_o.sum() > 0
    assert np.array_equal(r["gr"], gr_o.astype(np.float32))
    assert np.array_equal(r["psh"]["gr"], r["gr"][:, : o.num["GR"] // 10])
    # every ECTrialsData histogram, bit for bit (float sums included)
    for name, _ in cbmtest.TRIAL_PSH:
        assert cbmtest.same_values(r["psh"][name].ravel(), td["psh"][name].ravel()).all(), name
    # the rasters, over the rows the run fills (the reference leaves the
    # others as allocated)
    filled = cbmtest.raster_rows_filled(proto)
    for name, _ in cbmtest.TRIAL_RASTER:
        a, b = r["raster"][name], td["raster"][name]
        a, b = a.reshape(-1, a.shape[-1])[:filled], b.reshape(-1, b.shape[-1])
        assert np.array_equal(a, b[:filled]), name
        assert not b[filled:].any()
    # the protocol did something: CS trials spike NCs, move the eyelid and
    # fill the histograms and rasters
    assert nc.sum() > 0 and eye.max() > 0
    assert all(td["psh"][n].any() for n in ("go", "grInputGO", "goOutSynScale", "mf", "sc", "pc"))
    assert td["raster"]["go"].any() and td["raster"]["pc"].any()


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
def test_oracle_matches_reference_two_zones(tmp_path):
    """Two microzones and GO->GO wiring from the package's generator: zone 1
    takes its own plasticity steps and error drive (mzone.cpp:726-736,
    cbmsimcore.cpp:322-325), and both zones' records and final state must
    equal the reference's."""
    from cerebellum_simulation_b200 import networks
    net = networks.build_random_network(8, 6, 4, 4, 10, networks.act_params("16k"), seed=5, gr_per_go=128,
                                       mf_per_go=3, vel=40, gogo=((1, 1, 0.0),), n_zones=2)
    st = str(tmp_path / "z2.state")
    net.writeState(st)
    mf = cbmtest.counter_mf(1024, 600, 8, rate_hi=0.08)
    ev = {2: [("plast", 1, -0.003, 0.002)], 300: [("errdrive", 1, 1.0), ("errdrive", 0, 0.5)],
          450: [("plastreset", 1)]}
    fin_ref = str(tmp_path / "ref_final.state")
    ref = cbmtest.ref_run(st, mf, [3, 4], ev, final_path=fin_ref).reshape(600, -1)
    o = Oracle(st, seeds=[3, 4])
    tr = o.run(mf, ev)
    assert cbmtest.first_difference(ref, tr, o.num) is None
    fin = str(tmp_path / "oracle_final.state")
    o.save(fin)
    assert open(fin, "rb").read() == open(fin_ref, "rb").read()


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
def test_mf_population_estimate_matches_reference(tmp_path):
    """networks.MFPopulation.from_trial_data over the oracle's MF histogram
    equals the reference's ECMFPopulation(ECTrialsData *) over its own, bit
    for bit, and MFPopulation reads and writes the reference's file byte for
    byte."""
    from cerebellum_simulation_b200 import networks
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol()
    o = Oracle(st, seeds=[7])
    rates = cbmtest.protocol_rates(o.num["MF"], seed=1)
    steps = 3 * proto["trialSteps"]
    _, _, _, _, td = o.run_protocol(proto, rates, steps, record=False, trial_data=True)
    ref_path = str(tmp_path / "ref.mfpop")
    cbmtest.ref_run_protocol(st, proto, rates, steps, [7], mf_population=ref_path)
    ref = networks.MFPopulation.read(ref_path)
    got = networks.MFPopulation.from_trial_data(td["psh"]["mf"], proto["numDataTrials"], proto["binSteps"],
                                                proto["preCS"], proto["csOff"] - proto["csOn"])
    for a, b in ((got.bg, ref.bg), (got.cs_tonic, ref.cs_tonic), (got.cs_phasic, ref.cs_phasic)):
        assert cbmtest.same_values(a, b).all()
    # the estimate follows the rates the fibres were driven with (60 ms of
    # background per fibre, so only roughly)
    assert np.corrcoef(got.bg, rates[0])[0, 1] > 0.3 and got.cs_phasic.mean() > got.bg.mean()
    out = str(tmp_path / "rt.mfpop")
    ref.write(out)
    assert open(out, "rb").read() == open(ref_path, "rb").read()


@pytest.mark.parametrize("name", ["config2", "config3"])
def test_oracle_matches_reference_golden_large(tmp_path, name):
    """The 1M-GR network (32 PC x 32,768 PF: the reference's PF->PC reduction
    in its widest shape, 512 threads and 32 pair-adds each, kernels.cu:
    445-469, which the 16K networks never reach) over 1000 active steps in
    which plasticity moves PF->PC weights both ways, and the dense 4M-GR
    network (4096 GO, 128 PC) over 400: every trace record and the final
    state against the reference's, recorded by tests/golden/make_golden.py
    (inputs: cbmtest.golden_large_case)."""
    gold = cbmtest.load_json(name + "_digests.json")
    net, mf, ev = cbmtest.golden_large_case(name)
    st = str(tmp_path / "net.state")
    net.writeState(st)
    del net
    with open(st, "rb") as f:
        assert cbmtest.sha(np.frombuffer(f.read(), np.uint8)) == gold["initial_state"], \
            "network generator is not deterministic"
    steps = gold["steps"]
    assert mf.shape[0] == steps
    o = Oracle(st, seeds=[7])
    tr = o.run(mf, ev)
    assert tr.shape[1] == gold["record_bytes"]
    assert np.unpackbits(tr[:, : o.num["GR"] // 8], axis=1).sum() > 100000
    got = [cbmtest.sha(r) for r in tr]
    del tr
    bad = [i for i, (a, b) in enumerate(zip(got, gold["records"])) if a != b]
    assert not bad, f"first differing step {bad[0] + 1}"
    fin = str(tmp_path / "final.state")
    o.save(fin)
    with open(fin, "rb") as f:
        assert cbmtest.sha(np.frombuffer(f.read(), np.uint8)) == gold["final_state"]
    # the run exercises plasticity: the reference's final weights differ
    # from the initial ones, and the oracle's final state is the reference's
    assert gold["final_arrays"]["0/pfSynWeightPC"] != gold["initial_arrays"]["0/pfSynWeightPC"]
    import cerebellum_simulation_b200 as cbm
    w0, w1 = cbm.CBMState(st).array("pfSynWeightPC", 0), cbm.CBMState(fin).array("pfSynWeightPC", 0)
    assert (w1 < w0).any() and (w1 > w0).any()


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
def test_trial_data_file_matches_reference(tmp_path):
    """trialdata.write_ec_trials_data over the oracle's records writes the
    reference's ECTrialsData::writeData file byte for byte (a 280-step
    window, so every raster row is written by the run)."""
    from cerebellum_simulation_b200.trialdata import write_ec_trials_data
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol()
    o = Oracle(st, seeds=[7])
    rates = cbmtest.protocol_rates(o.num["MF"], seed=1)
    steps = 3 * proto["trialSteps"]
    tr, _, _, eye, td = o.run_protocol(proto, rates, steps, trial_data=True)
    ref_path, ref_session = str(tmp_path / "ref.data"), str(tmp_path / "ref.session")
    cbmtest.ref_run_protocol(st, proto, rates, steps, [7], data_file=ref_path, session_file=ref_session)
    ours = str(tmp_path / "ours.data")
    write_ec_trials_data(ours, td, cbmtest.gr_psh_from_trace(tr, proto, o.num["GR"]),
                         eye.reshape(proto["numDataTrials"], -1), proto, o.num["GR"])
    a, b = open(ours, "rb").read(), open(ref_path, "rb").read()
    assert len(a) == len(b) and a == b, next(i for i in range(min(len(a), len(b))) if a[i] != b[i])
    # the driver's session file (writeDataToFile): final state, then the data
    fin = str(tmp_path / "final.state")
    o.save(fin)
    assert open(ref_session, "rb").read() == open(fin, "rb").read() + a
    # and read back as the driver's resume constructor does
    from cerebellum_simulation_b200 import networks
    from cerebellum_simulation_b200.trialdata import read_session
    state, data = read_session(ref_session)
    assert state.getNumZones() == 1 and data["end"] == len(open(ref_session, "rb").read())
    for name, h in td["psh"].items():
        assert cbmtest.same_values(data["psh"][name].ravel(), h.ravel()).all(), name
    for name, r in td["raster"].items():
        assert np.array_equal(data["raster"][name], r), name
    pop = networks.MFPopulation.from_trial_data(data["psh"]["mf"], data["psh_trials"]["mf"], proto["binSteps"],
                                                data["header"]["msPreCS"], data["header"]["msCS"])
    assert pop.bg.shape == (o.num["MF"],) and np.isfinite(pop.rates()).all()


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
def test_eyelid_session_follows_the_driver(tmp_path):
    """EyelidSession (the driver's three constructors, run and
    writeDataToFile) drives a simulator through the calls the device tests
    check, with the protocol the driver uses; resuming from the reference's
    own session file gives the state and the MF tables the reference
    re-estimates from it."""
    from cerebellum_simulation_b200 import networks
    from cerebellum_simulation_b200.eyelid import EyelidSession
    st_path = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol()
    o = Oracle(st_path, seeds=[7])
    rates = cbmtest.protocol_rates(o.num["MF"], seed=1)
    steps = 3 * proto["trialSteps"]
    ref_session, ref_pop = str(tmp_path / "ref.session"), str(tmp_path / "ref.mfpop")
    cbmtest.ref_run_protocol(st_path, proto, rates, steps, [7], session_file=ref_session, mf_population=ref_pop)

    calls = []

    class FakeSim:
        def __init__(self, state, seeds, device=0):
            calls.append(("create", seeds, device))

        def __getattr__(self, name):
            return lambda *a, **k: calls.append((name, a, k))

    args = (7, 4, 400, 120, 260, 150, 1, 0, 3)
    s = EyelidSession.resume(ref_session, *args, sim_factory=FakeSim, preCS=60, postCS=80)
    want = networks.MFPopulation.read(ref_pop)
    assert np.array_equal(s.mf_population.rates(), want.rates())
    assert s.state.getNumZones() == 1 and s.state.con("numGR") == o.num["GR"]
    p = s.protocol
    assert (p["trialSteps"], p["csOn"], p["csOff"], p["csPhasicOff"], p["csStartTrial"], p["mfSeed"]) == \
        (400, 120, 260, 150, 1, 7)
    # the driver's LTD step: -0.0005 x ((csOff - csOn + msLTDStartAPIO) / msLTDDurationIO), at least 0.5
    ratio = max((140 + s.state.act("msLTDStartAPIO")) / s.state.act("msLTDDurationIO"), 0.5)
    assert p["plastLTD"] == pytest.approx(-0.0005 * ratio) and p["plastLTP"] == 0.0005
    s.run(chunk=50)
    s.write_data_to_file(str(tmp_path / "out.session"))
    names = [c[0] for c in calls]
    assert names == ["create", "set_eyelid_protocol", "record_gr", "record_trial_data", "run", "write_session"]
    assert calls[0][1] == [7] and calls[4][1] == (4 * 400,) and calls[4][2] == {"chunk": 50}
    assert np.array_equal(calls[1][1][0], want.rates()) and calls[1][2] == p
    assert calls[5][1] == (str(tmp_path / "out.session"), s.mf_population)
    # the file constructor reads the same tables back
    f = EyelidSession.from_files(st_path, ref_pop, *args, sim_factory=FakeSim)
    assert np.array_equal(f.mf_population.rates(), want.rates())


@pytest.mark.skipif(not os.path.exists(cbmtest.REF_STATEVAR), reason="reference harness oracle/_ref not built")
def test_state_variable_coding_matches_reference():
    """networks.StateVariableMF's rates equal the reference's StateVariable
    (Gaussian updates of 4 variables over ordered fibre shares, compiled from
    Matthew_Sim_CBM/includes/statevariable.hpp) bit for bit, over a stretch
    of the synthetic trajectory plus clamped and edge values."""
    import subprocess
    import tempfile
    from cerebellum_simulation_b200 import networks
    c = networks.StateVariableMF(1024, seed=4)
    vals = np.stack([c.values(t) for t in range(0, 3000, 37)]).astype(np.float32)
    vals[3] = np.float32([-5, 5, -1, 1])
    with tempfile.TemporaryDirectory() as d:
        for n, a in (("r", c.relaxed), ("e", c.excited), ("v", vals)):
            np.ascontiguousarray(a, np.float32).tofile(os.path.join(d, n))
        out = os.path.join(d, "o")
        subprocess.run([cbmtest.REF_STATEVAR, "1024", "4", repr(float(c.lo)), repr(float(c.hi)),
                        repr(float(c.gauss_width)), os.path.join(d, "r"), os.path.join(d, "e"), os.path.join(d, "v"),
                        str(len(vals)), out], check=True, capture_output=True)
        ref = np.fromfile(out, np.float32).reshape(len(vals), 1024)
    ours = np.stack([c.rates_for(v) for v in vals])
    assert np.array_equal(ref.view(np.uint32), ours.view(np.uint32))
    assert ours.max() > 39 and ours.min() < 10


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
def test_trials_data_getters_read_the_reference_file(tmp_path):
    """trialdata.TrialsData over the reference's own data file: the
    histograms' trial counts and bin widths, and the rasters' spike times
    (SpikeRasterBitArray::getCellSpikeTimes: bit 31 first, one step apart),
    which must be the window steps at which the oracle's trace has the cells
    spiking (time k is window step k + 1: the first update comes at window
    step 32 and covers steps 1-32)."""
    from cerebellum_simulation_b200.trialdata import TrialsData
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol()
    o = Oracle(st, seeds=[7])
    rates = cbmtest.protocol_rates(o.num["MF"], seed=1)
    steps = 3 * proto["trialSteps"]
    tr, _, _, eye, _ = o.run_protocol(proto, rates, steps, trial_data=True)
    ref_path = str(tmp_path / "ref.data")
    cbmtest.ref_run_protocol(st, proto, rates, steps, [7], data_file=ref_path)
    d = TrialsData.from_file(ref_path)
    rec_from = proto["csOn"] - proto["preCS"]
    rec_len = proto["csOff"] + proto["postCS"] - rec_from
    assert d.getMSTotal() == rec_len and d.getMaxNumTrials() == proto["numDataTrials"]
    assert d.getTSPerRasterUpdate() == 32
    go = d.getPSH("go")
    assert go.getNumTrials() == proto["numDataTrials"] and go.getBinWidthInMS() == proto["binSteps"]
    assert go.getNumBins() == -(-rec_len // proto["binSteps"]) and go.getNumCells() == o.num["GO"]
    # spike times from the trace, field by field
    off, fields = 0, {}
    for name, dt, cnt in cbmtest.record_layout(o.num):
        nb = np.dtype(dt).itemsize * cnt
        fields[name] = tr[:, off: off + nb].view(dt)
        off += nb
    rows = rec_len // 32
    seen = 0
    for name, key in (("pc", "apPC0"), ("go", "apGO"), ("nc", "apNC0")):
        raster = d.getRaster(name)
        for trial in range(proto["numDataTrials"]):
            first = (proto["dataStartTrial"] + trial) * proto["trialSteps"] + rec_from  # trace row of window step 0
            ap = fields[key][first + 1: first + 1 + 32 * rows]
            for cell in range(raster.getNumCells()):
                want = [int(k) for k in np.nonzero(ap[:, cell])[0]]
                assert raster.getCellSpikeTimes(cell, trial) == want, (name, trial, cell)
                seen += len(want)
        k = 37
        assert raster.getPopSpikesAtTS(k, 0) == [bool(v) for v in
                                                  fields[key][proto["dataStartTrial"] * proto["trialSteps"] + rec_from + k + 1]]
    assert seen > 100
    assert d.getEyelidData(0)[:3] == [float(v) for v in eye[:3]]


def test_oracle_step_rates_equal_protocol_tables(tmp_path):
    """The oracle's driver with per-step rate rows (the state-variable input's
    form) equals its driver with the protocol's tables when every row holds
    the background table and no trial has a CS."""
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.statevar_protocol(17)
    a = Oracle(st, seeds=[7])
    rates = cbmtest.protocol_rates(a.num["MF"], seed=3)
    a.run_protocol(proto, rates, 400, record=False)
    pa = str(tmp_path / "a.state")
    a.save(pa)
    b = Oracle(st, seeds=[7])
    b.run_protocol_step_rates(proto, np.stack([rates[0]] * 7), 400)
    pb = str(tmp_path / "b.state")
    b.save(pb)
    assert open(pa, "rb").read() == open(pb, "rb").read()
