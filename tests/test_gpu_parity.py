"""Parity of the B200 step with the CPU oracle (which is pinned to the
reference by tests/test_oracle_pin.py).

Spike rasters and every float state that spikes depend on must match bit for
bit; the GO glutamate/mGluR arrays, which no spike depends on, are compared
within FP_RTOL (they use the double-precision exp of two different math
libraries).  All calls go through the C ABI (libcbm_b200.so).
"""
import os

import numpy as np
import pytest

import cbmtest
from cbmtest import Oracle

pytestmark = pytest.mark.gpu

INNET_CON = ["haspGLfromMFtoGL", "pGLfromMFtoGL", "numpGLfromGLtoGO", "pGLfromGLtoGO", "numpGRfromMFtoGR",
             "pGRfromMFtoGR", "numpGRfromGOtoGR", "pGRfromGOtoGR", "numpGRfromGRtoGO", "pGRfromGRtoGO",
             "pGRDelayMaskfromGRtoGO", "pGRDelayMaskfromGRtoBSP", "numpMFfromMFtoGO", "pMFfromMFtoGO",
             "numpGOGABAOutGOGO", "pGOGABAOutGOGO"]
INNET_ACT = ["histMF", "apBufMF", "apGO", "apBufGO", "vGO", "vCoupleGO", "threshCurGO", "inputMFGO", "inputGOGO",
             "gMFGO", "gGRGO", "gGOGO", "gMGluRGO", "gMGluRIncGO", "mGluRGO", "gluGO", "apGR", "apBufGR",
             "gMFGR", "gMFSumGR", "gGOGR", "gGOSumGR", "threshGR", "vGR", "gKCaGR", "historyGR", "apSC",
             "apBufSC", "gPFSC", "threshSC", "vSC", "inputSumPFSC"]
ZONE_ACT = ["apBC", "apBufBC", "inputPCBC", "gPFBC", "gPCBC", "threshBC", "vBC", "apPC", "apBufPC", "inputBCPC",
            "inputSCPC", "pfSynWeightPC", "inputSumPFPC", "gPFPC", "gBCPC", "gSCPC", "vPC", "threshPC",
            "histPCPopAct", "apIO", "apBufIO", "inputNCIO", "gNCIO", "threshIO", "vIO", "vCoupleIO",
            "pfPCPlastTimerIO", "apNC", "apBufNC", "inputPCNC", "inputMFNC", "gPCNC", "gPCScaleNC",
            "mfSynWeightNC", "gmaxNMDAofMFtoNC", "gmaxAMPAofMFtoNC", "gMFNMDANC", "gMFAMPANC", "threshNC",
            "vNC", "synIOPReleaseNC"]


def compare_states(path_a, path_b):
    import cerebellum_simulation_b200 as cbm
    a, b = cbm.CBMState(path_a), cbm.CBMState(path_b)
    problems = []
    names = [(n, -1) for n in INNET_CON + INNET_ACT] + [(n, z) for z in range(a.getNumZones()) for n in ZONE_ACT]
    for n, z in names:
        x, y = a.array(n, z), b.array(n, z)
        if n in cbmtest.FP_TOLERANT_ARRAYS:
            if not np.allclose(x, y, rtol=cbmtest.FP_RTOL, atol=1e-30, equal_nan=True):
                problems.append(f"{n}: beyond rtol {cbmtest.FP_RTOL}")
        elif not cbmtest.same_values(x, y).all():
            problems.append(f"{n}[{z}]: {int(np.sum(~cbmtest.same_values(x, y)))} elements differ")
    return problems


def run_both(tmp_path, st_path, mf, seeds, events=None):
    import cerebellum_simulation_b200 as cbm
    o = Oracle(st_path, seeds=seeds)
    tr_o = o.run(mf, events)
    st = cbm.CBMState(st_path)
    sim = cbm.CBMSimCore(st, seeds, device=0)
    tr_p = cbmtest.product_run(sim, mf, events)
    fin_o, fin_p = str(tmp_path / "oracle.state"), str(tmp_path / "b200.state")
    o.save(fin_o)
    sim.writeToState(fin_p)
    return o, tr_o, tr_p, fin_o, fin_p


EVENTS = {
    5: [("plast", 0, -0.01, 0.005)],
    700: [("errdrive", 0, 1.0)],
    1000: [("errdrive", 0, 0.6)],
    1200: [("plastreset", 0)],
    1300: [("grgoinc", 0.01)],
    1400: [("grgoincreset",)],
}


def test_reference_network_16k_bit_exact(tmp_path):
    """The reference's own 16K network (its generator), 1500 steps with
    plasticity, error-drive and GR->GO gain events."""
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    mf = cbmtest.counter_mf(1024, 1500, 11)
    o, tr_o, tr_p, fo, fp = run_both(tmp_path, st, mf, [7], EVENTS)
    gold = cbmtest.load_json("ref16k_digests.json")
    assert [cbmtest.sha(r) for r in tr_o] == gold["records"]
    assert cbmtest.first_difference(tr_o, tr_p, o.num) is None
    assert compare_states(fo, fp) == []


def nc_offsets(num):
    """Byte offsets of each zone's NC spikes in a trace record (cbmtest.product_record's layout)."""
    off = num["GR"] // 8 + 9 * num["GO"] + 5 * num["SC"]
    per_zone = 5 * (num["BC"] + num["PC"] + num["IO"] + num["NC"])
    return [off + z * per_zone + 5 * (num["BC"] + num["PC"] + num["IO"]) for z in range(num["zones"])]


def test_nc_export_right_after_each_step(tmp_path):
    """exportAPNC called straight after each calcActivity, as a driver loop
    does (the NC spikes come through mapped host memory while the step's GR
    pass may still run), returns the oracle's NC spikes of that step, every
    step of 1500 on the reference's 16K network and of 600 in both zones of
    a two-zone network."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    st = cbmtest.golden_state("ref16k", str(tmp_path))
    two = networks.build_random_network(8, 6, 4, 4, 10, networks.act_params("16k"), seed=5, gr_per_go=128,
                                       mf_per_go=3, vel=40, gogo=((1, 1, 0.0),), n_zones=2)
    p2 = str(tmp_path / "two.state")
    two.writeState(p2)
    for path, steps, rate in ((st, 1500, None), (p2, 600, 0.08)):
        mf = cbmtest.counter_mf(1024, steps, 11) if rate is None else cbmtest.counter_mf(1024, steps, 8, rate_hi=rate)
        o = Oracle(path, seeds=[7, 8])
        tr = o.run(mf, EVENTS)
        offs = nc_offsets(o.num)
        sim = cbm.CBMSimCore(cbm.CBMState(path), [7, 8], device=0)
        zones = sim.getMZoneList()
        n_nc = o.num["NC"]
        spikes = 0
        for s in range(steps):
            for ev in EVENTS.get(s + 1, []):
                if ev[0] == "errdrive" and ev[1] < len(zones):
                    sim.updateErrDrive(ev[1], ev[2])
                elif ev[0] == "plast" and ev[1] < len(zones):
                    zones[ev[1]].setGRPCPlastSteps(ev[2], ev[3])
                elif ev[0] == "plastreset":
                    zones[ev[1]].resetGRPCPlastSteps()
                elif ev[0] == "grgoinc":
                    sim.getInputNet().setGIncGRtoGO(ev[1])
                elif ev[0] == "grgoincreset":
                    sim.getInputNet().resetGIncGRtoGO()
            sim.updateMFInput(mf[s])
            sim.calcActivity()
            for z, zone in enumerate(zones):
                got = zone.exportAPNC()
                want = tr[s, offs[z]:offs[z] + n_nc]
                assert np.array_equal(got, want), f"step {s + 1} zone {z}"
                spikes += int(want.sum())
        assert spikes > 0
        sim.close()


def test_config1_bit_exact(tmp_path):
    """Config 1: 16,384 GR with random wiring, 2000 steps of regenerating
    Poisson MF input at 1-30 Hz, PF->PC plasticity forced on."""
    from cerebellum_simulation_b200 import networks
    net = networks.config1_network(seed=0)
    p = str(tmp_path / "c1.state")
    net.writeState(p)
    mf = networks.uniform_mf_stream(1024, 2000, seed=0)
    ev = {1: [("plast", 0, -0.002, 0.001)], 1500: [("errdrive", 0, 1.0)]}
    o, tr_o, tr_p, fo, fp = run_both(tmp_path, p, mf, [3], ev)
    assert cbmtest.first_difference(tr_o, tr_p, o.num) is None
    assert compare_states(fo, fp) == []


def test_two_zones_bit_exact(tmp_path):
    from cerebellum_simulation_b200 import networks
    net = networks.build_random_network(8, 6, 4, 4, 10, networks.act_params("16k"), seed=5, gr_per_go=128,
                                       mf_per_go=3, vel=40, gogo=((1, 1, 0.0),), n_zones=2)
    p = str(tmp_path / "z2.state")
    net.writeState(p)
    mf = cbmtest.counter_mf(1024, 600, 8, rate_hi=0.08)
    ev = {2: [("plast", 1, -0.003, 0.002)], 300: [("errdrive", 1, 1.0), ("errdrive", 0, 0.5)]}
    o, tr_o, tr_p, fo, fp = run_both(tmp_path, p, mf, [3, 4], ev)
    assert cbmtest.first_difference(tr_o, tr_p, o.num) is None
    assert compare_states(fo, fp) == []


def test_config2_1m_bit_exact_short(tmp_path):
    """Config 2 size (1,048,576 GR, 1024 GO, 32 PC x 32,768 PF): 150 steps."""
    from cerebellum_simulation_b200 import networks
    net = networks.config2_network(seed=0)
    p = str(tmp_path / "c2.state")
    net.writeState(p)
    mf = networks.eyelid_mf_stream(1024, 150, seed=0, cs_on=50, cs_off=120)
    ev = {1: [("plast", 0, -0.0005, 0.0005)], 119: [("errdrive", 0, 1.0)]}
    o, tr_o, tr_p, fo, fp = run_both(tmp_path, p, mf, [9], ev)
    assert cbmtest.first_difference(tr_o, tr_p, o.num) is None
    assert compare_states(fo, fp) == []


def test_config3_4m_bit_exact_short(tmp_path):
    """Config 3 size (4,194,304 GR, 4096 GO x 1024 GR, 128 PC x 32,768 PF;
    its microzone arrays exceed shared memory, so the microzone CTA runs on
    global memory): 80 steps of state-variable-coded MF input."""
    from cerebellum_simulation_b200 import networks
    net = networks.config3_network(seed=0)
    p = str(tmp_path / "c3.state")
    net.writeState(p)
    mf = networks.config3_mf_stream(1024, 80, seed=0)
    ev = {1: [("plast", 0, -0.0005, 0.0005)], 60: [("errdrive", 0, 1.0)]}
    o, tr_o, tr_p, fo, fp = run_both(tmp_path, p, mf, [9], ev)
    assert cbmtest.first_difference(tr_o, tr_p, o.num) is None
    assert compare_states(fo, fp) == []


@pytest.mark.parametrize("name", ["config2", "config3"])
def test_chained_single_steps_equal_graph_runs(tmp_path, name):
    """Single steps queued without a synchronisation between them run as a
    chain of programmatic dependent launches (each small-cell kernel waits
    on the device for the previous step's GR pass, whose last CTA waits for
    its own step's small-cell kernel).  Such steps, on the 1M-GR network
    (the pass in one wave) and on the dense 4M-GR network (the pass in four
    waves), advance the network exactly as graph-chunk replays do."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    if name == "config2":
        net, n = networks.config2_network(seed=3), 240
        mf = networks.eyelid_mf_stream(1024, n, seed=3, cs_on=40, cs_off=200)
    else:
        net, n = networks.config3_network(seed=3), 60
        mf = networks.config3_mf_stream(1024, n, seed=3)
    p = str(tmp_path / "net.state")
    net.writeState(p)
    events = {2: [("plast", 0, -0.0005, 0.0005)], n // 2: [("errdrive", 0, 1.0)]}
    a = cbm.CBMSimCore(cbm.CBMState(p), [5], device=0)
    cbmtest.product_run(a, mf, events, record=False)
    fa = str(tmp_path / "a.state")
    a.writeToState(fa)
    b = cbm.CBMSimCore(cbm.CBMState(p), [5], device=0, resident_steps=n)
    b.load_mf_stream(cbm.mf_bits(mf, b.mf_words()))
    zone = b.getMZoneList()[0]
    t = 0
    for te in sorted(events):
        b.run(te - 1 - t, chunk=16)
        t = te - 1
        for ev in events[te]:
            if ev[0] == "plast":
                zone.setGRPCPlastSteps(ev[2], ev[3])
            else:
                b.updateErrDrive(ev[1], ev[2])
    b.run(n - t, chunk=16)
    assert b.steps_done() == n
    fb = str(tmp_path / "b.state")
    b.writeToState(fb)
    assert compare_states(fa, fb) == []


@pytest.mark.parametrize("name,vec", [("config2", "0"), ("config2", "1"), ("config3", "0")])
def test_large_networks_match_reference_golden(tmp_path, name, vec, monkeypatch):
    """The device against the reference itself, with no oracle in between:
    every step's spike raster and spike-relevant float state of the 1M-GR
    network over 1000 steps (PF->PC weights moving both ways from about step
    200) and of the dense 4M-GR network over 400, and every array of the
    final state, equal the digests of the reference's own run
    (tests/golden/make_golden.py; inputs cbmtest.golden_large_case).  The
    four GO glutamate/mGluR arrays, which no spike reads, are compared with
    the oracle in the tests above instead.  The 1M network runs with the
    default GR pass and with the vector pass."""
    import cerebellum_simulation_b200 as cbm
    monkeypatch.setenv("CBM_PASS_VEC", vec)
    gold = cbmtest.load_json(name + "_digests.json")
    net, mf, ev = cbmtest.golden_large_case(name)
    p = str(tmp_path / "net.state")
    net.writeState(p)
    del net
    sim = cbm.CBMSimCore(cbm.CBMState(p), [7], device=0)
    if vec == "1":
        assert sim.pass_geometry()[0] == "grPassVecKernel"
    zones, inet = sim.getMZoneList(), sim.getInputNet()
    for s in range(mf.shape[0]):
        for e in ev.get(s + 1, []):
            if e[0] == "plast":
                zones[e[1]].setGRPCPlastSteps(e[2], e[3])
            elif e[0] == "errdrive":
                sim.updateErrDrive(e[1], e[2])
        sim.updateMFInput(mf[s])
        sim.calcActivity()
        rec = cbmtest.product_record(sim, None)
        if cbmtest.sha(rec) != gold["records"][s]:
            pytest.fail(f"step {s + 1}: the device's record differs from the reference's")
    fin = str(tmp_path / "b200.state")
    sim.writeToState(fin)
    sim.close()
    got = cbmtest.state_array_digests(fin)
    bad = [k for k, v in gold["final_arrays"].items()
           if k.split("/")[1] not in cbmtest.FP_TOLERANT_ARRAYS and got[k] != v]
    assert not bad, f"final state arrays differ from the reference's: {bad}"
    assert gold["final_arrays"]["0/pfSynWeightPC"] != gold["initial_arrays"]["0/pfSynWeightPC"]


def test_graph_run_equals_step_calls(tmp_path):
    """Resident-input CUDA-graph runs give the step-by-step API's result."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    net = networks.config1_network(seed=1)
    p = str(tmp_path / "c1.state")
    net.writeState(p)
    mf = networks.uniform_mf_stream(1024, 700, seed=4)
    a = cbm.CBMSimCore(cbm.CBMState(p), [5], device=0)
    cbmtest.product_run(a, mf, record=False)
    fa = str(tmp_path / "a.state")
    a.writeToState(fa)
    b = cbm.CBMSimCore(cbm.CBMState(p), [5], device=0, resident_steps=700)
    b.load_mf_stream(cbm.mf_bits(mf, b.mf_words()))
    b.run(700, chunk=64)
    assert b.steps_done() == 700
    fb = str(tmp_path / "b.state")
    b.writeToState(fb)
    assert open(fa, "rb").read() == open(fb, "rb").read()


def test_flushed_runs_equal_graph_runs(tmp_path):
    """The measurement paths (each step alone after an L2 flush, and the
    same with the two kernels on separate streams) advance the network
    exactly as graph-chunk replays do."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    net = networks.config1_network(seed=2)
    p = str(tmp_path / "c1.state")
    net.writeState(p)
    mf = networks.uniform_mf_stream(1024, 240, seed=6)
    a = cbm.CBMSimCore(cbm.CBMState(p), [5], device=0, resident_steps=240)
    a.load_mf_stream(cbm.mf_bits(mf, a.mf_words()))
    a.run(240, chunk=40)
    fa = str(tmp_path / "a.state")
    a.writeToState(fa)
    b = cbm.CBMSimCore(cbm.CBMState(p), [5], device=0, resident_steps=240)
    b.load_mf_stream(cbm.mf_bits(mf, b.mf_words()))
    assert b.run_flushed(80, 1 << 20) > 0
    pass_ms, tail_ms = b.run_flushed_kernels(80, 1 << 20)
    assert pass_ms > 0 and tail_ms > 0
    b.run(80, chunk=40)
    assert b.steps_done() == 240
    fb = str(tmp_path / "b.state")
    b.writeToState(fb)
    assert open(fa, "rb").read() == open(fb, "rb").read()


def test_device_exp_matches_host_exp():
    """The double exponential of the GO glutamate update and the
    state-variable MF coding equals the host C library's exp (the
    reference's exp(double)) on every probed input: the whole finite range,
    the range the Gaussian coding and the glutamate term use, arguments
    whose results are subnormal, and the special values."""
    import ctypes
    import cerebellum_simulation_b200 as cbm
    rng = np.random.default_rng(1)
    x = np.concatenate([
        rng.uniform(-745, 710, 3_000_000), rng.uniform(-40, 0, 3_000_000), rng.uniform(-1, 1, 1_000_000),
        rng.uniform(-760, -700, 500_000), rng.uniform(-1e-12, 1e-12, 100_000),
        (rng.integers(0, 2**63, 1_000_000, dtype=np.uint64) | (rng.integers(0, 2, 1_000_000, dtype=np.uint64) << 63)
         ).view(np.float64),
        np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 709.78, 709.79, -745.13, -745.14, -708.4, 512.0, -512.0,
                  1024.0, -1024.0, 2.0 ** -60, -2.0 ** -60])])
    dev = cbm.device_exp(x)
    lib = Oracle.lib()
    lib.cbm_oracle_exp_array.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    host = np.empty_like(x)
    lib.cbm_oracle_exp_array(x.ctypes.data, host.ctypes.data, x.size)
    same = (dev.view(np.uint64) == host.view(np.uint64)) | (np.isnan(dev) & np.isnan(host))
    assert same.all(), f"{int((~same).sum())} mismatches, first at x={x[~same][0]!r}"


def test_device_expf_matches_host_expf():
    """The small-cell updates' float exponential equals the host C library's
    expf (the reference's exp(float)) on every probed input."""
    import ctypes
    import cerebellum_simulation_b200 as cbm
    rng = np.random.default_rng(0)
    x = np.concatenate([
        rng.uniform(-110, 95, 4_000_000).astype(np.float32),
        rng.uniform(-2, 2, 4_000_000).astype(np.float32),
        (rng.integers(0, 2**32, 4_000_000, dtype=np.uint64).astype(np.uint32)).view(np.float32),
        np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 88.0, 88.7228, 88.72284, -103.97, -103.9721, -104.0,
                  1e-30, -1e-30, float.fromhex('0x1.04845ep+5'), float.fromhex('-0x1.f8cbb2p+5')], dtype=np.float32)])
    dev = cbm.device_expf(x)
    lib = Oracle.lib()
    lib.cbm_oracle_expf_array.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    host = np.empty_like(x)
    lib.cbm_oracle_expf_array(x.ctypes.data, host.ctypes.data, x.size)
    same = (dev.view(np.uint32) == host.view(np.uint32)) | (np.isnan(dev) & np.isnan(host))
    assert same.all(), f"{int((~same).sum())} mismatches, first at x={x[~same][0]!r}"
