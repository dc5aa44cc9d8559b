"""Batched instances (cbm_batch_*): networks of different sizes, seeds and
parameters advanced together, each under its own device protocol, give for
every instance the records and final state the oracle gives for that
instance alone; the autotuner's switch of GR-pass kernel keeps that."""
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
    assert kind in (0, 1) and ms > 0
    b.run(2 * protos[0]["trialSteps"] - 150, 50)
    _check_instances(b, [cbmtest.golden_state("ref16k", str(tmp_path))] + paths[1:], protos, rates,
                     2 * protos[0]["trialSteps"], tmp_path, "b")
