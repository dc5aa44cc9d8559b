"""Batched instances (cbm_batch_*): networks of different sizes, seeds and
parameters advanced together, each under its own device protocol, give for
every instance the records and final state the oracle gives for that
instance alone; the autotuner's switch of GR-pass kernel keeps that."""
import os

import numpy as np
import pytest

import cbmtest
from cbmtest import Oracle
from test_gpu_parity import compare_states

pytestmark = pytest.mark.gpu


def _instances(tmp_path):
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    paths = []
    paths.append(cbmtest.golden_state("ref16k", str(tmp_path)))
    st = networks.config1_network(seed=9)
    st.setActParam("threshBaseGO", st.act("threshBaseGO") * 1.1)
    p = str(tmp_path / "c1.state"); st.writeState(p); paths.append(p)
    st = networks.build_random_network(9, 8, 5, 5, 10, networks.act_params("dense"), seed=6,
                                       go_out_per_gr=4, mf_per_go=16, vel=147)
    p = str(tmp_path / "n131k.state"); st.writeState(p); paths.append(p)
    protos = [cbmtest.short_protocol(mfSeed=31 + i, plastLTD=-0.004 * (0.5 + i), numDataTrials=2)
              for i in range(len(paths))]
    return paths, protos


def _oracle_instance(path, proto, rates, steps, seed, out):
    o = Oracle(path, seeds=[seed])
    _, nc, pc, eye = o.run_protocol(proto, rates, steps, record=False)
    o.save(out)
    return nc, pc, eye


def _check_instances(b, paths, protos, rates, steps, tmp_path, tag):
    for i, p in enumerate(paths):
        nc, pc, eye = _oracle_instance(p, protos[i], rates[i], steps, 40 + i, str(tmp_path / f"o{i}_{tag}.state"))
        assert np.array_equal(b.trial_record(i, "nc").ravel(), nc), f"instance {i}"
        assert np.array_equal(b.trial_record(i, "pc").ravel(), pc), f"instance {i}"
        assert cbmtest.same_values(b.trial_record(i, "eyelid").ravel(), eye).all(), f"instance {i}"
        fin = str(tmp_path / f"b{i}_{tag}.state")
        b.writeToState(i, fin)
        assert compare_states(str(tmp_path / f"o{i}_{tag}.state"), fin) == [], f"instance {i}"


def test_batch_matches_instances_alone(tmp_path):
    import cerebellum_simulation_b200 as cbm
    paths, protos = _instances(tmp_path)
    states = [cbm.CBMState(p) for p in paths]
    rates = [cbmtest.protocol_rates(st.con("numMF"), seed=10 + i) for i, st in enumerate(states)]
    b = cbm.CBMBatch(states, [[40 + i] for i in range(len(states))], device=0)
    for i in range(len(states)):
        b.set_eyelid_protocol(i, rates[i], **protos[i])
    steps = 2 * protos[0]["trialSteps"]
    b.run(steps, 40)
    assert b.num_gr() == sum(st.con("numGR") for st in states)
    _check_instances(b, paths, protos, rates, steps, tmp_path, "a")


def test_batch_autotune_keeps_results(tmp_path):
    import cerebellum_simulation_b200 as cbm
    paths, protos = _instances(tmp_path)
    states = [cbm.CBMState(p) for p in paths]
    rates = [cbmtest.protocol_rates(st.con("numMF"), seed=10 + i) for i, st in enumerate(states)]
    b = cbm.CBMBatch(states, [[40 + i] for i in range(len(states))], device=0)
    for i in range(len(states)):
        b.set_eyelid_protocol(i, rates[i], **protos[i])
    b.run(150, 50)
    choice, ms = b.autotune(50)
    kind = int(choice.split(",")[0])
    assert kind in (0, 1, 3) and ms > 0
    b.run(2 * protos[0]["trialSteps"] - 150, 50)
    _check_instances(b, [cbmtest.golden_state("ref16k", str(tmp_path))] + paths[1:], protos, rates,
                     2 * protos[0]["trialSteps"], tmp_path, "b")


def test_batch_config4_sizes_match_instances_alone(tmp_path):
    """Instances at the batched sweep's sizes, built as its workload builds
    them (random wiring with 4 GO targets per GR, 1024 GO, 32 PC, GO
    threshold and LTD step scaled per instance): 2,097,152 GR (32 PC x 65,536
    PF), 1,048,576 GR (the shape-specialised pass's network shape) and
    262,144 GR, advanced together in one batch over two 400-step trials
    whose second trial moves PF->PC weights.  Each instance's records and
    final state equal the oracle's for that instance alone."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    paths, protos = [], []
    for i, (gx, gy, go_scale, ltd_scale) in enumerate([(11, 10, 0.9, 1.6), (11, 9, 1.1, 0.7), (10, 8, 1.0, 1.0)]):
        st = networks.build_random_network(gx, gy, 6, 4, 10, networks.act_params("dense"), seed=70 + i,
                                           go_out_per_gr=4, mf_per_go=16, vel=147)
        st.setActParam("threshBaseGO", st.act("threshBaseGO") * go_scale)
        p = str(tmp_path / f"inst{i}.state")
        st.writeState(p)
        del st
        paths.append(p)
        protos.append(cbmtest.short_protocol(mfSeed=51 + i, plastLTD=-0.004 * ltd_scale, numDataTrials=2))
    states = [cbm.CBMState(p) for p in paths]
    assert [s.con("numGR") for s in states] == [1 << 21, 1 << 20, 1 << 18]
    rates = [cbmtest.protocol_rates(st.con("numMF"), seed=20 + i) for i, st in enumerate(states)]
    b = cbm.CBMBatch(states, [[40 + i] for i in range(len(states))], device=0)
    for i in range(len(states)):
        b.set_eyelid_protocol(i, rates[i], **protos[i])
    steps = 2 * protos[0]["trialSteps"]
    b.run(steps, 50)
    _check_instances(b, paths, protos, rates, steps, tmp_path, "c4")
    for i, p in enumerate(paths):
        w0 = cbm.CBMState(p).array("pfSynWeightPC", 0)
        w1 = cbm.CBMState(str(tmp_path / f"b{i}_c4.state")).array("pfSynWeightPC", 0)
        assert (w1 != w0).any(), f"instance {i}: no PF->PC weight moved"


def test_batch_trial_data_matches_instances_alone(tmp_path):
    """ECTrialsData recorded for batch instances (cbm_batch_record_trial_data:
    one kernel over every recording instance after each step) equals the
    oracle's records of each instance alone, histograms (float sums
    included) and rasters; an instance that does not record stays without
    records."""
    import cerebellum_simulation_b200 as cbm
    paths, protos = _instances(tmp_path)
    states = [cbm.CBMState(p) for p in paths]
    rates = [cbmtest.protocol_rates(st.con("numMF"), seed=10 + i) for i, st in enumerate(states)]
    b = cbm.CBMBatch(states, [[40 + i] for i in range(len(states))], device=0)
    for i in range(len(states)):
        b.set_eyelid_protocol(i, rates[i], **protos[i])
    for i in (0, 2):
        b.record_trial_data(i)
    steps = 2 * protos[0]["trialSteps"]
    b.run(steps, 40)
    for i in (0, 2):
        o = Oracle(paths[i], seeds=[40 + i])
        _, _, _, _, want = o.run_protocol(protos[i], rates[i], steps, record=False, trial_data=True)
        got = b.trial_data(i)
        for name, a in want["psh"].items():
            assert cbmtest.same_values(got["psh"][name].ravel(), a.ravel()).all(), (i, name)
        for name, a in want["raster"].items():
            assert np.array_equal(got["raster"][name], a), (i, name)
        assert want["psh"]["go"].any() and want["raster"]["go"].any()
    with pytest.raises(cbm.CBMError):
        b.trial_data(1)


def _vec_batch(paths, protos, rates, steps, vec_env, tmp_path, tag):
    """Run a batch with CBM_PASS_VEC set as given at its construction; the
    pass kernel in use, every instance's records and final state bytes."""
    import cerebellum_simulation_b200 as cbm
    old = os.environ.get("CBM_PASS_VEC")
    os.environ["CBM_PASS_VEC"] = vec_env
    try:
        b = cbm.CBMBatch([cbm.CBMState(p) for p in paths], [[60 + i] for i in range(len(paths))], device=0)
    finally:
        if old is None:
            del os.environ["CBM_PASS_VEC"]
        else:
            os.environ["CBM_PASS_VEC"] = old
    for i in range(len(paths)):
        b.set_eyelid_protocol(i, rates[i], **protos[i])
    b.run(steps, 50)
    out = []
    for i in range(len(paths)):
        fin = str(tmp_path / f"{tag}{i}.state")
        b.writeToState(i, fin)
        with open(fin, "rb") as f:
            out.append((b.trial_record(i, "nc").copy(), b.trial_record(i, "pc").copy(),
                        b.trial_record(i, "eyelid").copy(), f.read()))
    kind = b.pass_geometry()[0]
    b.close()
    return kind, out


def test_batch_vector_pass_matches_per_tile_pass(tmp_path):
    """The batched vector pass (one persistent launch whose warps claim
    128-cell units across every instance; each instance's previous-step
    PF->PC reduction spread over the CTAs) gives every instance the records
    and final state, bit for bit, that the batch's per-tile pass gives (the
    per-tile pass is pinned to the oracle above): 131,072, 262,144 and
    524,288 GR of the eyelid shape with different GO thresholds and LTD
    steps, two 400-step trials moving PF->PC weights."""
    from cerebellum_simulation_b200 import networks
    import cerebellum_simulation_b200 as cbm
    paths, protos = [], []
    for i, (gx, gy, go_scale, ltd_scale) in enumerate([(9, 8, 1.0, 1.0), (10, 8, 0.9, 1.5), (10, 9, 1.1, 0.6)]):
        st = networks.build_random_network(gx, gy, 5, 5, 10, networks.act_params("dense"), seed=80 + i,
                                           go_out_per_gr=4, mf_per_go=16, vel=147)
        st.setActParam("threshBaseGO", st.act("threshBaseGO") * go_scale)
        p = str(tmp_path / f"v{i}.state")
        st.writeState(p)
        del st
        paths.append(p)
        protos.append(cbmtest.short_protocol(mfSeed=71 + i, plastLTD=-0.004 * ltd_scale, numDataTrials=2))
    rates = [cbmtest.protocol_rates(cbm.CBMState(p).con("numMF"), seed=30 + i) for i, p in enumerate(paths)]
    steps = 2 * protos[0]["trialSteps"]
    kind_vec, got = _vec_batch(paths, protos, rates, steps, "1", tmp_path, "vec")
    kind_tile, want = _vec_batch(paths, protos, rates, steps, "0", tmp_path, "tile")
    assert kind_vec == "grPassVecBatchKernel" and kind_tile == "grPassTmaKernel"
    for i in range(len(paths)):
        for k, name in enumerate(("nc", "pc", "eyelid")):
            assert np.array_equal(got[i][k], want[i][k]), (i, name)
        assert got[i][3] == want[i][3], f"instance {i}: final state differs"
        w0 = cbm.CBMState(paths[i]).array("pfSynWeightPC", 0)
        w1 = cbm.CBMState(str(tmp_path / f"vec{i}.state")).array("pfSynWeightPC", 0)
        assert (w1 != w0).any(), f"instance {i}: no PF->PC weight moved"
