"""Every compiled geometry of the two TMA GR passes, the per-tile pass both
specialised for the network's shape and not, and the vector pass, give the same network
state, bit for bit, as the plain GR pass kernel (the plain kernel is pinned
to the oracle by test_gpu_parity.py): the per-tile pass (consumer warps x
rows per warp x stages x resident CTAs x slot bound) and the persistent pass
(consumer warps x stages x resident CTAs x slot bound).  The microzone CTA's
global-memory mode (networks whose arrays do not fit in shared memory) gives
the same state as its staged mode."""
import os

import numpy as np
import pytest

import cbmtest

pytestmark = pytest.mark.gpu

TILE_GEOMETRIES = ["8,1,3,2,4", "8,1,3,3,4", "8,1,4,2,4", "8,1,2,3,4", "4,1,4,4,4", "4,2,3,3,4", "4,2,4,2,4",
                   "4,2,2,4,4", "8,1,3,2,0", "4,1,4,1,0", "2,1,4,1,0", "1,1,4,1,0"]
PERSISTENT_GEOMETRIES = ["4,4,2,4", "4,3,3,4", "2,4,4,4", "2,6,3,4", "4,4,2,0", "2,4,2,0", "1,4,2,0"]
# 8,2,2,4 (16-row units) does not fit tiles of 8 rows
EVENTS = {1: [("plast", 0, -0.002, 0.002)], 60: [("errdrive", 0, 1.0)], 90: [("grgoinc", 0.01)]}


def run_with(env, state_path, mf, out_path):
    import cerebellum_simulation_b200 as cbm
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        sim = cbm.CBMSimCore(cbm.CBMState(state_path), [3], device=0)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    cbmtest.product_run(sim, mf, EVENTS, record=False)
    sim.writeToState(out_path)
    sim.close()
    with open(out_path, "rb") as f:
        return f.read()


def test_tma_pass_geometries_match_plain_pass(tmp_path):
    from cerebellum_simulation_b200 import networks
    # 131,072 GR, 32 PCs of 4096 fibres: tiles of 8 rows x 32 cells; 4 MF,
    # 3 GO and 4 GR->GO slots per cell
    st = networks.build_random_network(9, 8, 5, 5, 10, networks.act_params("dense"), seed=5,
                                       go_out_per_gr=4, mf_per_go=16, vel=147)
    path = str(tmp_path / "net.state")
    st.writeState(path)
    mf = networks.uniform_mf_stream(1024, 120, seed=5, lo=5.0, hi=60.0)
    want = run_with({"CBM_PASS_TMA": "0"}, path, mf, str(tmp_path / "plain.state"))
    for g in TILE_GEOMETRIES:
        # this network has the eyelid shape: slot bound 4 runs the
        # shape-specialised kernel, CBM_PASS_SHAPE=0 the run-time-shape one
        for shape_env in ({}, {"CBM_PASS_SHAPE": "0"}) if g.endswith(",4") else ({},):
            env = {"CBM_PASS_TMA": g, "CBM_PASS_PERSIST": "0", **shape_env}
            got = run_with(env, path, mf, str(tmp_path / f"tma_{g}.state"))
            assert got == want, f"per-tile geometry {g} {shape_env} differs from the plain pass"
    for g in PERSISTENT_GEOMETRIES:
        got = run_with({"CBM_PASS_PERSIST": g}, path, mf, str(tmp_path / f"persist_{g}.state"))
        assert got == want, f"persistent geometry {g} differs from the plain pass"
    # the vector pass (four cells per lane, claimed work, PF->PC running
    # sums from the previous step's pair sums), and the default
    for claim in ("1", "2", "4"):
        got = run_with({"CBM_PASS_VEC": "1", "CBM_VEC_CLAIM": claim}, path, mf, str(tmp_path / f"vec{claim}.state"))
        assert got == want, f"the vector pass ({claim} units per claim) differs from the plain pass"
    got = run_with({}, path, mf, str(tmp_path / "default.state"))
    assert got == want, "the default pass differs from the plain pass"


def test_pass_kind_selection(tmp_path):
    """Single networks of the eyelid shape run the per-tile pass by default
    and the vector pass with CBM_PASS_VEC=1; a 16K network whose SC blocks
    hold 32 cells never runs the vector pass."""
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    st = networks.build_random_network(9, 8, 5, 5, 10, networks.act_params("dense"), seed=5,
                                       go_out_per_gr=4, mf_per_go=16, vel=147)
    path = str(tmp_path / "net.state")
    st.writeState(path)

    def kind_with(env, p):
        old = {k: os.environ.get(k) for k in env}
        os.environ.update(env)
        try:
            sim = cbm.CBMSimCore(cbm.CBMState(p), [3], device=0)
        finally:
            for k, v in old.items():
                if v is None:
                    del os.environ[k]
                else:
                    os.environ[k] = v
        kind = sim.pass_geometry()[0]
        sim.close()
        return kind

    assert kind_with({}, path) == "grPassTmaKernel"
    assert kind_with({"CBM_PASS_VEC": "1"}, path) == "grPassVecKernel"
    small = networks.config1_network(seed=1)
    p16 = str(tmp_path / "c1.state")
    small.writeState(p16)
    assert kind_with({"CBM_PASS_VEC": "1"}, p16) != "grPassVecKernel"


def test_zone_global_memory_mode_matches_staged(tmp_path):
    from cerebellum_simulation_b200 import networks
    st = networks.build_random_network(9, 8, 5, 5, 10, networks.act_params("dense"), seed=6,
                                       go_out_per_gr=4, mf_per_go=16, vel=147)
    path = str(tmp_path / "net.state")
    st.writeState(path)
    mf = networks.uniform_mf_stream(1024, 120, seed=6, lo=5.0, hi=60.0)
    want = run_with({}, path, mf, str(tmp_path / "staged.state"))
    got = run_with({"CBM_ZONE_STAGE": "0"}, path, mf, str(tmp_path / "global.state"))
    assert got == want, "the microzone CTA's global-memory mode differs from its staged mode"
