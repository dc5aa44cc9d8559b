"""Trials driven on the device (cbm_sim_set_eyelid_protocol): MF generation,
US, PF->PC plasticity window, eyelid integrator and trial records against
the oracle's restatement of the reference's eyelid driver (pinned to the
reference's PoissonRegenCells / EyelidIntegrator in test_oracle_pin.py)."""
import numpy as np
import pytest

import cbmtest
from cbmtest import Oracle
from test_gpu_parity import compare_states

pytestmark = pytest.mark.gpu


def _oracle(state_path, proto, rates, steps, tmp_path):
    o = Oracle(state_path, seeds=[7])
    tr, nc, pc, eye = o.run_protocol(proto, rates, steps)
    fin = str(tmp_path / "oracle.state")
    o.save(fin)
    return o, tr, nc, pc, eye, fin


def _compare_records(sim, o_nc, o_pc, o_eye):
    nc, pc, eye = sim.trial_record("nc"), sim.trial_record("pc"), sim.trial_record("eyelid")
    assert np.array_equal(nc.ravel(), o_nc)
    assert np.array_equal(pc.ravel(), o_pc)
    assert cbmtest.same_values(eye.ravel(), o_eye).all()
    return nc, eye


def test_protocol_step_by_step_bit_exact(tmp_path):
    import cerebellum_simulation_b200 as cbm
    st_path = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol()
    st = cbm.CBMState(st_path)
    rates = cbmtest.protocol_rates(st.con("numMF"), seed=1)
    steps = 3 * proto["trialSteps"]
    o, tr_o, o_nc, o_pc, o_eye, fin_o = _oracle(st_path, proto, rates, steps, tmp_path)
    sim = cbm.CBMSimCore(st, [7], device=0)
    sim.set_eyelid_protocol(rates, **proto)
    for s in range(steps):
        sim.calcActivity()
        rec = cbmtest.product_record(sim, None)
        if not cbmtest.same_values(rec, tr_o[s]).all():
            pytest.fail(f"step {s + 1}: " + cbmtest.first_difference(rec, tr_o[s], o.num))
    nc, eye = _compare_records(sim, o_nc, o_pc, o_eye)
    assert nc.sum() > 0 and eye.max() > 0
    fin_p = str(tmp_path / "b200.state")
    sim.writeToState(fin_p)
    assert compare_states(fin_o, fin_p) == []


def test_protocol_graph_replay_bit_exact(tmp_path):
    """Whole trials replayed as CUDA graphs, the protocol started after some
    host-driven steps."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    st = networks.config1_network(seed=4)
    st_path = str(tmp_path / "c1.state")
    st.writeState(st_path)
    proto = cbmtest.short_protocol(trialSteps=300, csOn=80, csOff=200, csPhasicOff=80, csStartTrial=0,
                                   numDataTrials=2, dataStartTrial=1, mfSeed=23)
    rates = cbmtest.protocol_rates(st.con("numMF"), seed=2)
    lead = cbmtest.counter_mf(st.con("numMF"), 37, 5)
    steps = 3 * proto["trialSteps"]
    o = Oracle(st_path, seeds=[7])
    o.run(lead)
    _, o_nc, o_pc, o_eye = o.run_protocol(proto, rates, steps, record=False)
    fin_o = str(tmp_path / "oracle.state")
    o.save(fin_o)
    sim = cbm.CBMSimCore(cbm.CBMState(st_path), [7], device=0)
    cbmtest.product_run(sim, lead, record=False)
    sim.set_eyelid_protocol(rates, **proto)
    sim.run(steps, 50)
    _compare_records(sim, o_nc, o_pc, o_eye)
    fin_p = str(tmp_path / "b200.state")
    sim.writeToState(fin_p)
    assert compare_states(fin_o, fin_p) == []
    with pytest.raises(cbm.CBMError):
        sim.updateMFInput(np.zeros(st.con("numMF"), dtype=np.uint8))


def test_gr_histogram_matches_oracle_spikes(tmp_path):
    """The device GR peri-stimulus histogram (cbm_sim_record_gr) equals the
    oracle's GR spikes counted over the recording windows of the kept trials,
    both under graph replay and step by step."""
    import cerebellum_simulation_b200 as cbm
    st_path = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol(dataStartTrial=1, numDataTrials=2)
    st = cbm.CBMState(st_path)
    rates = cbmtest.protocol_rates(st.con("numMF"), seed=2)
    steps = 3 * proto["trialSteps"]
    o = Oracle(st_path, seeds=[7])
    tr, _, _, _ = o.run_protocol(proto, rates, steps)
    # the rule test_oracle_pin.py pins to the reference's PeriStimHistFloat
    want = cbmtest.gr_psh_from_trace(tr, proto, st.con("numGR"))
    assert want.sum() > 0
    for replay in (True, False):
        sim = cbm.CBMSimCore(cbm.CBMState(st_path), [7], device=0)
        sim.set_eyelid_protocol(rates, **proto)
        sim.record_gr()
        if replay:
            sim.run(steps, chunk=100)
        else:
            for _ in range(steps):
                sim.calcActivity()
        got = sim.trial_record("gr")
        sim.close()
        assert got.dtype == np.uint16 and got.shape == want.shape
        assert np.array_equal(got.astype(np.uint32), want), f"replay={replay}"


@pytest.mark.parametrize("window,replay", [(dict(), True), (dict(preCS=56, postCS=60), False)])
def test_trial_data_matches_oracle(tmp_path, window, replay):
    """The device ECTrialsData records (cbm_sim_record_trial_data), recorded
    together with the GR histogram, equal the oracle's (pinned to the
    reference's ECTrialsData in test_oracle_pin.py) bit for bit: every
    histogram, float sums included, and every raster, under graph replay and
    step by step; the 256-step window makes the raster trials drift."""
    import cerebellum_simulation_b200 as cbm
    st_path = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol(**window)
    st = cbm.CBMState(st_path)
    rates = cbmtest.protocol_rates(st.con("numMF"), seed=1)
    steps = 3 * proto["trialSteps"]
    o = Oracle(st_path, seeds=[7])
    tr, _, _, o_eye, want = o.run_protocol(proto, rates, steps, trial_data=True)
    sim = cbm.CBMSimCore(cbm.CBMState(st_path), [7], device=0)
    sim.set_eyelid_protocol(rates, **proto)
    sim.record_gr()
    sim.record_trial_data()
    if replay:
        sim.run(steps, chunk=100)
    else:
        for _ in range(steps):
            sim.calcActivity()
    got = sim.trial_data()
    gr = sim.trial_record("gr")
    sim.write_trial_data(str(tmp_path / "device.data"))
    sim.close()
    for name, a in want["psh"].items():
        assert got["psh"][name].shape == a.shape, name
        assert cbmtest.same_values(got["psh"][name].ravel(), a.ravel()).all(), name
    for name, a in want["raster"].items():
        assert np.array_equal(got["raster"][name], a), name
    assert np.array_equal(gr.astype(np.uint32), cbmtest.gr_psh_from_trace(tr, proto, st.con("numGR")))
    smooth = cbm.eyelid_out(o_eye.reshape(proto["numDataTrials"], -1))
    assert cbmtest.same_values(got["eyelid"].ravel(), smooth.ravel()).all()
    # the driver's data file from the device equals the one from the oracle's
    # records (which test_oracle_pin.py holds to the reference's file)
    from cerebellum_simulation_b200.trialdata import write_ec_trials_data
    write_ec_trials_data(str(tmp_path / "oracle.data"), want, cbmtest.gr_psh_from_trace(tr, proto, st.con("numGR")),
                         o_eye.reshape(proto["numDataTrials"], -1), proto, st.con("numGR"))
    assert open(tmp_path / "device.data", "rb").read() == open(tmp_path / "oracle.data", "rb").read()
    assert want["psh"]["go"].any() and want["raster"]["go"].any() and want["psh"]["mf"].any()


def test_eyelid_session_matches_oracle(tmp_path):
    """EyelidSession (the driver's trial loop and writeDataToFile) on the
    device: its session file holds the oracle's final state and, byte for
    byte, the data file of the oracle's records; its MF tables file holds
    the tables it ran with."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    from cerebellum_simulation_b200.eyelid import EyelidSession
    from cerebellum_simulation_b200.trialdata import read_session, write_ec_trials_data
    st_path = cbmtest.golden_state("ref16k", str(tmp_path))
    proto = cbmtest.short_protocol()
    n_trials = 3
    rates = cbmtest.protocol_rates(cbm.CBMState(st_path).con("numMF"), seed=1)
    pop = networks.MFPopulation(*rates)
    fixed = ("trialSteps", "csOn", "csOff", "csPhasicOff", "csStartTrial", "dataStartTrial", "numDataTrials", "mfSeed")
    s = EyelidSession(cbm.CBMState(st_path), pop, 7, n_trials, proto["trialSteps"], proto["csOn"], proto["csOff"],
                      proto["csPhasicOff"], proto["csStartTrial"], proto["dataStartTrial"], proto["numDataTrials"],
                      **{k: v for k, v in proto.items() if k not in fixed})
    s.run(chunk=100)
    out = str(tmp_path / "device.session")
    s.write_data_to_file(out)
    s.sim.close()
    o = Oracle(st_path, seeds=[7])
    tr, _, _, eye, td = o.run_protocol(s.protocol, rates, n_trials * proto["trialSteps"], trial_data=True)
    fin = str(tmp_path / "oracle.state")
    o.save(fin)
    state, data = read_session(out)
    dev_state = str(tmp_path / "device.state")
    state.writeState(dev_state)
    assert compare_states(fin, dev_state) == []
    odata = str(tmp_path / "oracle.data")
    n_gr = state.con("numGR")
    write_ec_trials_data(odata, td, cbmtest.gr_psh_from_trace(tr, s.protocol, n_gr),
                         eye.reshape(proto["numDataTrials"], -1), s.protocol, n_gr)
    raw, want = open(out, "rb").read(), open(odata, "rb").read()
    assert raw.endswith(want) and data["end"] == len(raw)
    assert np.array_equal(networks.MFPopulation.read(out + "_MFPop").rates(), pop.rates())


def test_config2_1m_full_trial_bit_exact(tmp_path):
    """A whole eyelid trial of the 1M-GR network (1,048,576 GR, 32 PC x 32,768
    PF: the benchmark's network and the widest PF->PC reduction) run on the
    device as graph replays: 5000 steps, CS at 2000-2500 ms, the US at step
    2499, LTD/LTP steps in force from 2200 to 2700 ms.  History bit 39 is set
    200 steps after a GR's first spiking bin, so plasticity moves PF->PC
    weights in this trial.  The final state (every GR array, every PF->PC
    weight), the NC/PC records, the eyelid trace and the ECTrialsData
    histograms and rasters equal the oracle's bit for bit, and weights have
    moved both down (LTD) and up (LTP)."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    st = networks.config2_network(seed=2)
    st_path = str(tmp_path / "c2.state")
    st.writeState(st_path)
    bg, cs = networks.eyelid_mf_rates(st.con("numMF"), seed=2)
    rates = np.stack([bg, cs, cs])
    proto = cbm.eyelid_protocol_defaults(st, mfSeed=5, numDataTrials=1)
    steps = proto["trialSteps"]
    assert steps == 5000 and proto["csOn"] == 2000 and proto["csOff"] == 2500
    o = Oracle(st_path, seeds=[7])
    _, o_nc, o_pc, o_eye, want = o.run_protocol(proto, rates, steps, record=False, trial_data=True)
    fin_o = str(tmp_path / "oracle.state")
    o.save(fin_o)
    sim = cbm.CBMSimCore(cbm.CBMState(st_path), [7], device=0)
    sim.set_eyelid_protocol(rates, **proto)
    sim.record_trial_data()
    sim.run(steps, 50)
    _compare_records(sim, o_nc, o_pc, o_eye)
    got = sim.trial_data()
    fin_p = str(tmp_path / "b200.state")
    sim.writeToState(fin_p)
    sim.close()
    assert compare_states(fin_o, fin_p) == []
    for name, a in want["psh"].items():
        assert cbmtest.same_values(got["psh"][name].ravel(), a.ravel()).all(), name
    for name, a in want["raster"].items():
        assert np.array_equal(got["raster"][name], a), name
    w0 = cbm.CBMState(st_path).array("pfSynWeightPC", 0)
    w1 = cbm.CBMState(fin_p).array("pfSynWeightPC", 0)
    assert (w1 < w0).sum() > 0 and (w1 > w0).sum() > 0, "no PF->PC weight moved both ways"
    assert o_pc.sum() > 0


def test_statevar_rates_match_host_coding(tmp_path):
    """The device's state-variable MF coding (cbm_sim_set_statevar_input)
    gives, row by row, the rates of networks.StateVariableMF (pinned to the
    reference's StateVariable::gaussMFAct in test_oracle_pin.py) bit for bit:
    the benchmark's coding (width 0.2 of the range) and a narrow one whose
    Gaussian underflows far from a fibre's preferred value, with values that
    leave the range (clamped)."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    st = networks.config1_network(seed=2)
    p = str(tmp_path / "c1.state")
    st.writeState(p)
    sim = cbm.CBMSimCore(cbm.CBMState(p), [7], device=0)
    for coding in (networks.StateVariableMF(1024, seed=3), networks.StateVariableMF(1024, seed=4, gauss_width=0.05)):
        vals = coding.trajectory(1500)
        vals[::97] *= 1.3  # some rows outside [lo, hi]
        sim.set_statevar_input(coding, vals, mfSeed=9)
        for r in range(0, vals.shape[0], 7):
            got = sim.statevar_rates(r)
            want = coding.rates_for(vals[r])
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"row {r}"
    sim.close()


def test_statevar_input_matches_oracle(tmp_path):
    """A network driven by the device's state-variable MF input (the dense
    configuration's coding) under graph replay ends in the oracle's state,
    bit for bit, when the oracle's generator takes the host coding's rates
    step by step; the input rows are reused cyclically."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    st = networks.build_random_network(9, 8, 5, 5, 10, networks.act_params("dense"), seed=8,
                                       go_out_per_gr=4, mf_per_go=16, vel=147)
    p = str(tmp_path / "net.state")
    st.writeState(p)
    coding = networks.StateVariableMF(1024, seed=5)
    vals = coding.trajectory(250)
    steps = 600
    rates = np.stack([coding.rates_for(v) for v in vals])
    o = Oracle(p, seeds=[7])
    o.run_protocol_step_rates(cbmtest.statevar_protocol(13), rates, steps)
    fin_o = str(tmp_path / "oracle.state")
    o.save(fin_o)
    sim = cbm.CBMSimCore(cbm.CBMState(p), [7], device=0)
    sim.set_statevar_input(coding, vals, mfSeed=13)
    sim.run(steps, 50)
    fin_p = str(tmp_path / "b200.state")
    sim.writeToState(fin_p)
    sim.close()
    assert compare_states(fin_o, fin_p) == []
    a = cbm.CBMState(fin_p).array("apBufMF")
    assert a.any(), "no MF spiked"
