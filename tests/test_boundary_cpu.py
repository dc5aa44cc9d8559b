"""CPU checks of the boundary: the C-ABI library loads and exports every
function the headers in include/ declare, state files round-trip byte for byte
through the reference format, and malformed input fails with an error code."""
import ctypes
import os
import re

import numpy as np
import pytest

import cbmtest

ROOT = cbmtest.ROOT


def declared_functions():
    names = set()
    for h in ("cbm_b200.h", "cbm_surrogate.h"):
        with open(os.path.join(ROOT, "include", h)) as f:
            text = f.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(cbm_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import cerebellum_simulation_b200 as cbm
    names = declared_functions()
    assert len(names) >= 30
    lib = ctypes.CDLL(cbm.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_state_roundtrip_reference_file(tmp_path):
    import cerebellum_simulation_b200 as cbm
    p = cbmtest.golden_state("ref16k", str(tmp_path))
    s = cbm.CBMState(p)
    assert s.getNumZones() == 1
    assert s.con("numGR") == 16384 and s.con("numGO") == 1024 and s.con("numpPCfromGRtoPC") == 512
    out = str(tmp_path / "rt.state")
    s.writeState(out)
    assert open(p, "rb").read() == open(out, "rb").read()


def test_loader_rebuilds_pc_to_bc_wiring(tmp_path):
    """The reference's file holds pBCfromPCtoBC where pPCfromPCtoBC belongs;
    the loader rebuilds pPCfromPCtoBC with connectPCtoBC's formula."""
    import cerebellum_simulation_b200 as cbm
    s = cbm.CBMState(cbmtest.golden_state("ref16k", str(tmp_path)))
    npc, nbc = s.con("numPC"), s.con("numBC")
    got = s.array("pPCfromPCtoBC", 0).reshape(npc, 16)
    want = np.array([[((i * (nbc // npc) - 6 + j) % nbc + nbc) % nbc for j in range(16)] for i in range(npc)])
    assert np.array_equal(got, want)


def test_derived_parameters():
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import networks
    s = networks.config1_network(seed=0)
    assert s.con("numGR") == 16384 and s.con("numGO") == 256 and s.con("numBC") == 128 and s.con("numSC") == 512
    # gLeak = raw/(6-dt), decays exp(-dt/tau) in float (activityparams.cpp:499-519)
    raw = s.act("rawGLeakGR")
    assert s.act("gLeakGR") == pytest.approx(raw / 5.0, rel=1e-7)
    assert s.act("gDecMFtoGR") == float(np.float32(np.exp(np.float32(-1) / np.float32(s.act("gMFDecayTGR")))))
    assert s.act("tsPerHistBinGR") == 5


@pytest.mark.parametrize("damage", ["truncate", "header"])
def test_malformed_state_file_is_rejected(tmp_path, damage):
    import cerebellum_simulation_b200 as cbm
    p = cbmtest.golden_state("ref16k", str(tmp_path))
    data = open(p, "rb").read()
    bad = str(tmp_path / "bad.state")
    with open(bad, "wb") as f:
        f.write(data[: len(data) // 2] if damage == "truncate" else b"1\nfoo 3\n")
    with pytest.raises(cbm.CBMError) as e:
        cbm.CBMState(bad)
    assert e.value.code == 4


def test_missing_state_file_is_an_io_error(tmp_path):
    import cerebellum_simulation_b200 as cbm
    with pytest.raises(cbm.CBMError) as e:
        cbm.CBMState(str(tmp_path / "nope.state"))
    assert e.value.code == 3


def test_mf_bits_packing():
    import cerebellum_simulation_b200 as cbm
    x = np.zeros((2, 1024), np.uint8)
    x[0, 0] = 1
    x[0, 33] = 1
    x[1, 1023] = 1
    b = cbm.mf_bits(x, 33)
    assert b.shape == (2, 33)
    assert b[0, 0] == 1 and b[0, 1] == 2 and b[1, 31] == 1 << 31 and b[1, 32] == 0


def test_cpp_facade_compiles_and_loads_a_reference_state(tmp_path):
    """include/cbm_core.hpp keeps the reference's class names; a driver
    written against them builds and loads a reference state file."""
    import subprocess
    exe = cbmtest.build_facade_check(str(tmp_path))
    p = cbmtest.golden_state("ref16k", str(tmp_path))
    out = subprocess.run([exe, p], check=True, capture_output=True, text=True).stdout
    assert "zones 1" in out
    lines = {l.split()[0]: l.split()[1:] for l in out.splitlines()}
    s = __import__("cerebellum_simulation_b200").CBMState(p)
    assert lines["cells"] == [str(s.con(n)) for n in ("numGR", "numGO", "numMF", "numSC", "numBC", "numPC",
                                                       "numNC", "numIO")] + ["ms", "1"]
    n_con, n_act, _, ltd, _, set_ok, ltd2, _, bad = lines["params"]
    assert int(n_con) > 20 and int(n_act) > 80 and set_ok == "1" and bad == "0"
    assert float(ltd2) == pytest.approx(2 * float(ltd))
    assert lines["gr0"][1] == str(int(s.array("numpGRfromMFtoGR")[0]))
    assert lines["gr0"][3] == str(int(s.array("numpGRfromGOtoGR")[0]))
    assert lines["gr0"][6] == str(int(s.array("numpGOfromGRtoGO")[0]))
    # the reference network has no GO->GO pairs and room for one per GO: the
    # pair goes to the end of both lists, and its removal empties them again
    # (a second removal finds nothing)
    assert lines["gogo"] == ["0", "0", "add", "1", "1", "1", "last", "1", "del", "1", "again", "0", "0", "0"]
    w = lines["weights"]
    assert int(w[0]) == 16384 and float(w[1]) == 0.25
    assert float(w[3]) == pytest.approx(s.act("initSynWofGRtoPC")) and w[5] == "1"


def _damage(s, name):
    """One out-of-range entry in a reference network's wiring."""
    if name == "pGRfromMFtoGR":
        assert s.array("numpGRfromMFtoGR")[0] >= 1
        s.array(name)[0] = s.con("numMF")
    elif name == "numpGRfromGOtoGR":
        s.array(name)[5] = s.con("maxnumpGRfromGOtoGR") + 1
    elif name == "pGRfromGRtoGO":
        g = int(np.argmax(s.array("numpGRfromGRtoGO") > 0))
        s.array(name)[g * s.con("maxnumpGRfromGRtoGO")] = s.con("numGO")
    elif name == "pGRDelayMaskfromGRtoGO":
        g = int(np.argmax(s.array("numpGRfromGRtoGO") > 0))
        s.array(name)[g * s.con("maxnumpGRfromGRtoGO")] = 3
    elif name == "numpGOCoupInGOGO":
        s.array(name)[7] = s.con("maxnumpGOCoupInGOGO") + 1
    elif name == "pBCfromBCtoPC":
        s.array(name, 0)[0] = s.con("numPC")


@pytest.mark.parametrize("name,code,words", [
    ("pGRfromMFtoGR", 5, "MF->GR index"),
    ("numpGRfromGOtoGR", 5, "GO->GR count"),
    ("pGRfromGRtoGO", 5, "GR->GO index"),
    ("pGRDelayMaskfromGRtoGO", 6, "one bit"),
    ("numpGOCoupInGOGO", 5, "GO coupling"),
    ("pBCfromBCtoPC", 5, "microzone"),
])
def test_malformed_network_is_rejected_before_the_device(tmp_path, name, code, words):
    """Every connectivity count and index is checked on the host when the
    simulator is created, before any device work, so the kernels carry no
    bounds checks and a bad network never reaches a GPU."""
    import cerebellum_simulation_b200 as cbm
    s = cbm.CBMState(cbmtest.golden_state("ref16k", str(tmp_path)))
    _damage(s, name)
    with pytest.raises(cbm.CBMError) as e:
        cbm.CBMSimCore(s, [7])
    assert e.value.code == code and words in str(e.value), str(e.value)


def test_valid_network_needs_a_device(tmp_path):
    """Without a GPU the simulator fails loudly (CBM_ERR_CUDA): there is no
    CPU fallback behind the API."""
    import cerebellum_simulation_b200 as cbm
    s = cbm.CBMState(cbmtest.golden_state("ref16k", str(tmp_path)))
    try:
        sim = cbm.CBMSimCore(s, [7])
    except cbm.CBMError as e:
        assert e.code == 2, str(e)
    else:
        sim.close()


def test_cpp_facade_state_in_a_stream_with_trailing_data(tmp_path):
    """CBMState::writeState(fstream&) then other data into one stream, and
    CBMState(fstream&) reading the state back and leaving the stream where
    the data starts, as the eyelid driver's session file is written and
    resumed (ecmanagementdelay.cpp:26-50, 275-290).  The state read back from
    the stream saves to the same bytes as the original file."""
    import subprocess
    exe = cbmtest.build_facade_check(str(tmp_path))
    p = cbmtest.golden_state("ref16k", str(tmp_path))
    out_path = str(tmp_path / "session")
    out = subprocess.run([exe, p, "--stream", out_path], check=True, capture_output=True, text=True).stdout
    assert "stream zones 1 trailer trailer 4242" in out
    state_bytes = open(p, "rb").read()
    session = open(out_path, "rb").read()
    assert session[: len(state_bytes)] == state_bytes
    assert session[len(state_bytes):] == b"trailer 4242\n"
    assert open(out_path + ".again", "rb").read() == state_bytes


def test_state_memory_calls_reject_a_small_buffer(tmp_path):
    """cbm_state_save_mem reports the state's size for a NULL buffer and
    refuses one that is too small; cbm_state_load_mem reports the bytes it
    consumed when data follows the state."""
    import ctypes
    import cerebellum_simulation_b200 as cbm
    lib = cbm.lib
    p = cbmtest.golden_state("ref16k", str(tmp_path))
    st = cbm.CBMState(p)
    size = ctypes.c_uint64()
    lib.cbm_state_save_mem.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                       ctypes.POINTER(ctypes.c_uint64)]
    assert lib.cbm_state_save_mem(st._h, None, 0, ctypes.byref(size)) == 0
    want = open(p, "rb").read()
    assert size.value == len(want)
    small = ctypes.create_string_buffer(16)
    assert lib.cbm_state_save_mem(st._h, small, 16, ctypes.byref(size)) == 1  # CBM_ERR_ARG
    buf = ctypes.create_string_buffer(size.value)
    assert lib.cbm_state_save_mem(st._h, buf, size.value, ctypes.byref(size)) == 0
    assert buf.raw == want
    data = want + b"next"
    h, used = ctypes.c_void_p(), ctypes.c_uint64()
    lib.cbm_state_load_mem.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                       ctypes.POINTER(ctypes.c_void_p)]
    assert lib.cbm_state_load_mem(data, len(data), ctypes.byref(used), ctypes.byref(h)) == 0
    assert used.value == len(want)
    lib.cbm_state_free(h)
    assert lib.cbm_state_load_mem(data[: len(want) // 2], len(want) // 2, ctypes.byref(used), ctypes.byref(h)) != 0


def test_python_state_accessors_match_the_facade(tmp_path):
    """The Python mirror of the state library's accessors gives what the C++
    facade's do on the same state file."""
    import subprocess
    import cerebellum_simulation_b200 as cbm
    exe = cbmtest.build_facade_check(str(tmp_path))
    p = cbmtest.golden_state("ref16k", str(tmp_path))
    lines = {l.split()[0]: l.split()[1:]
             for l in subprocess.run([exe, p], check=True, capture_output=True, text=True).stdout.splitlines()}
    s = cbm.CBMState(p)
    cp, ap, con = s.getConnectivityParams(), s.getActivityParams(), s.getInnetConState()
    assert lines["cells"][:8] == [str(f()) for f in (cp.getNumGR, cp.getNumGO, cp.getNumMF, cp.getNumSC,
                                                     cp.getNumBC, cp.getNumPC, cp.getNumNC, cp.getNumIO)]
    assert int(lines["cells"][9]) == ap.getMSPerTimeStep()
    assert int(lines["params"][0]) == len(cp.getParamCopy()) and int(lines["params"][1]) == len(ap.getParamCopy())
    ltd = ap.getParam("grPCLTDDecIO")
    assert float(lines["params"][3]) == pytest.approx(ltd)
    assert ap.setParam("grPCLTDDecIO", 2 * ltd) and not ap.setParam("noSuchParam", 1.0)
    assert ap.getParam("grPCLTDDecIO") == pytest.approx(2 * ltd) and ap.getParam("noSuchParam") == 0.0
    assert lines["gr0"] == ["mf", str(len(con.getpGRfromMFtoGR(0))), "go", str(len(con.getpGRfromGOtoGR(0))),
                            "go0", "gr", str(len(con.getpGOfromGRtoGOCon(0))), "incomplete",
                            str(len(con.getGRIncompIndfromGRtoGO()))]
    assert con.getpGRPopfromMFtoGR()[5] == con.getpGRfromMFtoGR(5)
    assert con.addGOGOConPair(0, 1) and not con.addGOGOConPair(0, 2)
    assert con.getpGOOutGOGOCon(0) == [1] and con.getpGOInGOGOCon(1) == [0]
    assert con.deleteGOGOConPair(0, 1) and not con.deleteGOGOConPair(0, 1)
    assert con.getpGOOutGOGOCon(0) == [] and con.getpGOInGOGOCon(1) == []
    z = s.getMZoneActState(0)
    s.array("pfSynWeightPC", 0)[0] = 0.25
    assert z.getGRPCSynWeightLinear()[0] == np.float32(0.25)
    z.resetGRPCSynWeight()
    assert np.all(z.getGRPCSynWeightLinear() == np.float32(s.act("initSynWofGRtoPC")))
    assert s.equivalent(cbm.CBMState(p))


@pytest.mark.parametrize("config", ["config1_network", "config2_network"])
def test_oracle_built_network_equals_the_products(tmp_path, config):
    """The oracle's restatement of CBMState(actPF, conPF, nZones) (initial
    values and microzone wiring, cbm_oracle_new) with the package's random
    input-net wiring writes the same state file, byte for byte, as the
    product's state library: the benchmark's CPU baseline builds its network
    this way, without the product's library."""
    import filecmp
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_state import OracleState
    from cerebellum_simulation_b200 import networks
    fn = getattr(networks, config)
    a, b = tmp_path / "product.state", tmp_path / "oracle.state"
    fn(seed=5).writeState(str(a))
    fn(seed=5, new_state=OracleState.new).writeState(str(b))
    assert filecmp.cmp(a, b, shallow=False)


def test_device_exp_table_is_the_mathematical_one():
    """kExpTab of the device's double exp holds, for k < 128, the tail
    (2^(k/128) - H) / H and asuint64(H) - (k << 45), with H = 2^(k/128)
    rounded to the nearest double: regenerated here at 80-digit precision
    and compared entry by entry with the table in the kernel source."""
    import struct
    from decimal import Decimal, getcontext
    src = open(os.path.join(ROOT, "cerebellum_simulation_b200", "csrc", "cbm_kernels.cu")).read()
    body = src[src.index("kExpTab[256] = {"):]
    body = body[body.index("{") + 1: body.index("};")]
    got = [int(v, 16) for v in re.findall(r"0x([0-9a-f]+)ull", body)]
    assert len(got) == 256
    getcontext().prec = 80
    ln2 = Decimal(2).ln()
    for k in range(128):
        v = (ln2 * k / 128).exp()
        h = float(v)
        tail = float((v - Decimal(h)) / Decimal(h))
        hb = struct.unpack("<Q", struct.pack("<d", h))[0]
        tb = struct.unpack("<Q", struct.pack("<d", tail))[0]
        assert got[2 * k] == tb and got[2 * k + 1] == (hb - (k << 45)) % 2 ** 64, k



def test_reference_generator_reproduces_the_reference_network(tmp_path):
    """CBMState(actPF, conPF, nZones, innetCRSeed, mzoneCRSeed, mzoneARSeed)
    with the reference's generator (cbm_state_generate, the C++ facade's
    constructor with the reference's signature): the 16K parameter files
    and seeds 11 / 22 / 33 give the reference's own state file
    (tests/golden/ref16k.state.xz, written by the reference's CBMState with
    the same arguments), byte for byte."""
    import lzma
    import subprocess
    import cerebellum_simulation_b200 as cbm
    params = os.path.join(ROOT, "cerebellum_simulation_b200", "params")
    act, con = os.path.join(params, "act_16k.txt"), os.path.join(params, "con_16k.txt")
    want = lzma.open(os.path.join(ROOT, "tests", "golden", "ref16k.state.xz")).read()
    st = cbm.CBMState.generate(open(con).read(), open(act).read(), 1, 11, [22], [33])
    out = tmp_path / "py.state"
    st.writeState(str(out))
    assert out.read_bytes() == want
    exe = cbmtest.build_facade_check(str(tmp_path))
    out2 = tmp_path / "cpp.state"
    r = subprocess.run([exe, "--generate", act, con, str(out2)], check=True, capture_output=True, text=True)
    assert "generated zones 1" in r.stdout
    assert out2.read_bytes() == want


@pytest.mark.skipif(not cbmtest.ref_available(), reason="reference harness oracle/_ref not built")
@pytest.mark.parametrize("zones,seeds", [(2, (5, 7, 9)), (1, (123456, 99, 1))])
def test_reference_generator_matches_the_reference_live(tmp_path, zones, seeds):
    """The same against the reference's generator run live (oracle/_ref/
    ref_gen) with other seeds and two microzones, whose PC->NC wiring draws
    from each zone's seed."""
    import subprocess
    import cerebellum_simulation_b200 as cbm
    params = os.path.join(ROOT, "cerebellum_simulation_b200", "params")
    act, con = os.path.join(params, "act_16k.txt"), os.path.join(params, "con_16k.txt")
    ref = tmp_path / "ref.state"
    subprocess.run([cbmtest.REF_GEN, act, con, str(zones), str(seeds[0]), str(seeds[1]), str(seeds[2]), str(ref)],
                   check=True, capture_output=True)
    st = cbm.CBMState.generate(open(con).read(), open(act).read(), zones, seeds[0],
                               [seeds[1] + z for z in range(zones)], [seeds[2] + z for z in range(zones)])
    out = tmp_path / "b200.state"
    st.writeState(str(out))
    assert out.read_bytes() == ref.read_bytes()
