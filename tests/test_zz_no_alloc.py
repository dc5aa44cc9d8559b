"""The allocation-free PF->PC sum entry point (cbm_pfpc_sums_noalloc).

It serves callers that cannot let the library allocate device memory during
a call (their framework owns all device memory through its own pool, or they
run a real-time loop that cannot absorb an allocation).  Here it
is checked through the C ABI against the simulator's own PF->PC input sums
(cbm_sim_write_to_state's inputSumPFPC), bit for bit, on two calls in a row,
and its size limit is checked.  This file runs last so that a failure here
leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

import cbmtest

pytestmark = pytest.mark.gpu


def _entry():
    import cerebellum_simulation_b200 as cbm
    fn = cbm.lib.cbm_pfpc_sums_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                   ctypes.c_void_p, ctypes.c_void_p]
    return fn


def _noalloc_sums(apbuf, mask, w, num_pc):
    import torch
    fn = _entry()
    d_ap = torch.from_numpy(apbuf.view(np.int32).copy()).cuda()
    d_mask = torch.from_numpy(mask.view(np.int32).copy()).cuda()
    d_w = torch.from_numpy(w.copy()).cuda()
    out = torch.full((num_pc,), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = fn(d_ap.data_ptr(), d_mask.data_ptr(), d_w.data_ptr(), apbuf.size, num_pc, out.data_ptr(), None)
    assert rc == 0, _last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _last_error():
    import cerebellum_simulation_b200 as cbm
    return cbm.lib.cbm_last_error().decode()


@pytest.mark.parametrize("shape", ["16k_rows512", "131k_rows4096"])
def test_noalloc_matches_simulator_sums_twice(tmp_path, shape):
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    if shape == "16k_rows512":
        # the reference generator's 16K network: 32 PCs of 512 fibres
        st = cbm.CBMState(cbmtest.golden_state("ref16k", str(tmp_path)))
        mf = cbmtest.counter_mf(1024, 400, 11)
    else:
        st = networks.build_random_network(9, 8, 5, 5, 10, networks.act_params("dense"), seed=2,
                                           go_out_per_gr=4, mf_per_go=16, vel=147)
        mf = networks.uniform_mf_stream(1024, 400, seed=2, lo=5.0, hi=60.0)
    num_pc = st.con("numPC")
    sim = cbm.CBMSimCore(st, [5], device=0)
    events = {1: [("plast", 0, -0.001, 0.001)], 150: [("errdrive", 0, 1.0)]}
    mask = st.array("pGRDelayMaskfromGRtoBSP").copy()
    zone = sim.getMZoneList()[0]
    t = 0
    for stop in (250, 380):  # two calls in a row, at two points of the run
        cbmtest.product_run(sim, mf[t:stop - 1], events, t0=t, record=False)
        apbuf = sim.getInputNet().exportAPBufGR()
        w = zone.exportPFPCWeights()
        got = _noalloc_sums(apbuf, mask, w, num_pc)
        # the simulator's sum of the same spikes and weights is the PC input
        # after one more step (two-phase pipeline, cbmsimcore.cpp:153, 215)
        cbmtest.product_run(sim, mf[stop - 1:stop], events, t0=stop - 1, record=False)
        sim.writeToState()
        want = st.array("inputSumPFPC", 0).copy()
        assert np.count_nonzero(want) > 0
        assert cbmtest.same_values(got, want).all(), (got[:4], want[:4])
        t = stop


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    fn = _entry()
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    # 256 rows of 16384 fibres need 256 x 512 partials > CBM_NOALLOC_MAX_PARTIALS
    rc = fn(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 1 << 22, 256, buf.data_ptr(), None)
    assert rc == 1
    assert "CBM_NOALLOC_MAX_PARTIALS" in _last_error()
