"""Test helpers: the CPU oracle (oracle/libcbm_oracle.so), the reference
harness (oracle/_ref/ref_run) and trace records of the B200 simulator in the
oracle's record layout."""
import ctypes
import hashlib
import json
import lzma
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "libcbm_oracle.so")
REF_RUN = os.path.join(ORACLE_DIR, "_ref", "ref_run")
REF_GEN = os.path.join(ORACLE_DIR, "_ref", "ref_gen")
REF_STATEVAR = os.path.join(ORACLE_DIR, "_ref", "ref_statevar")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def ensure_oracle():
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", ORACLE_DIR, "oracle"], check=True, capture_output=True)
    return ORACLE_LIB


class Oracle:
    """ctypes view of the C oracle (oracle/cbm_oracle.h)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(ensure_oracle())
            P, S, I, U, F = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_uint, ctypes.c_float
            lib.cbm_oracle_load.restype = P
            lib.cbm_oracle_load.argtypes = [S, S, ctypes.c_size_t]
            lib.cbm_oracle_free.argtypes = [P]
            lib.cbm_oracle_set_seeds.argtypes = [P, P]
            lib.cbm_oracle_update_err_drive.argtypes = [P, U, F]
            lib.cbm_oracle_set_plast_steps.argtypes = [P, U, F, F]
            lib.cbm_oracle_reset_plast_steps.argtypes = [P, U]
            lib.cbm_oracle_set_ginc_grgo.argtypes = [P, F]
            lib.cbm_oracle_reset_ginc_grgo.argtypes = [P]
            lib.cbm_oracle_run.argtypes = [P, P, ctypes.c_uint64, P]
            lib.cbm_oracle_trace_record_bytes.restype = ctypes.c_size_t
            lib.cbm_oracle_trace_record_bytes.argtypes = [P]
            lib.cbm_oracle_save.restype = I
            lib.cbm_oracle_save.argtypes = [P, S]
            lib.cbm_oracle_num.restype = ctypes.c_uint32
            lib.cbm_oracle_num.argtypes = [P, S]
            lib.cbm_oracle_protocol_sizes.argtypes = [P, P, P, P, P]
            lib.cbm_oracle_run_protocol.argtypes = [P, P, P, ctypes.c_uint64, P, P, P, P, P, P]
            lib.cbm_oracle_trial_data_sizes.argtypes = [P, P, P, P]
            lib.cbm_oracle_run_protocol_step_rates.argtypes = [P, P, P, ctypes.c_uint64, ctypes.c_uint64, P, P, P, P]
            cls._lib = lib
        return cls._lib

    def __init__(self, state_path, seeds=None):
        lib = self.lib()
        err = ctypes.create_string_buffer(256)
        self.h = lib.cbm_oracle_load(os.fsencode(state_path), err, 256)
        if not self.h:
            raise RuntimeError(err.value.decode())
        if seeds is not None:
            s = np.asarray(seeds, dtype=np.int32)
            lib.cbm_oracle_set_seeds(self.h, s.ctypes.data)
        self.rb = lib.cbm_oracle_trace_record_bytes(self.h)
        self.num = {k: lib.cbm_oracle_num(self.h, k.encode()) for k in ("GR", "GO", "MF", "SC", "BC", "PC", "NC", "IO", "zones")}

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().cbm_oracle_free(self.h)
            self.h = None

    def apply(self, ev):
        lib = self.lib()
        k = ev[0]
        if k == "errdrive":
            lib.cbm_oracle_update_err_drive(self.h, ev[1], ev[2])
        elif k == "plast":
            lib.cbm_oracle_set_plast_steps(self.h, ev[1], ev[2], ev[3])
        elif k == "plastreset":
            lib.cbm_oracle_reset_plast_steps(self.h, ev[1])
        elif k == "grgoinc":
            lib.cbm_oracle_set_ginc_grgo(self.h, ev[1])
        elif k == "grgoincreset":
            lib.cbm_oracle_reset_ginc_grgo(self.h)

    def run(self, mf, events=None, t0=0):
        """Steps t0+1 .. t0+len(mf); events maps 1-based step -> list of events."""
        mf = np.ascontiguousarray(mf, dtype=np.uint8)
        steps = mf.shape[0]
        tr = np.zeros((steps, self.rb), dtype=np.uint8)
        lib = self.lib()
        for s in range(steps):
            for ev in (events or {}).get(t0 + s + 1, []):
                self.apply(ev)
            row = np.ascontiguousarray(mf[s])
            lib.cbm_oracle_run(self.h, row.ctypes.data, 1, tr[s].ctypes.data)
        return tr

    def run_protocol(self, proto, rates, nsteps, record=True, trial_data=False):
        """The eyelid driver around nsteps steps (cbm_oracle_run_protocol):
        (trace, ncPSH, pcPSH, eyelid), and with trial_data the eyelid driver's
        ECTrialsData records as a dict (split_trial_data)."""
        lib = self.lib()
        p = ProtocolStruct.from_dict(proto)
        sizes = [ctypes.c_uint64() for _ in range(3)]
        lib.cbm_oracle_protocol_sizes(self.h, ctypes.byref(p), *[ctypes.byref(x) for x in sizes])
        nc = np.zeros(sizes[0].value, dtype=np.uint32)
        pc = np.zeros(sizes[1].value, dtype=np.uint32)
        eye = np.zeros(sizes[2].value, dtype=np.float32)
        psh = raster = None
        if trial_data:
            ts = [ctypes.c_uint64() for _ in range(2)]
            lib.cbm_oracle_trial_data_sizes(self.h, ctypes.byref(p), *[ctypes.byref(x) for x in ts])
            psh = np.zeros(ts[0].value, dtype=np.float32)
            raster = np.zeros(ts[1].value, dtype=np.uint32)
        rates = np.ascontiguousarray(rates, dtype=np.float32)
        tr = np.zeros((nsteps, self.rb), dtype=np.uint8) if record else None
        lib.cbm_oracle_run_protocol(self.h, ctypes.byref(p), rates.ctypes.data, nsteps,
                                    tr.ctypes.data if record else None, nc.ctypes.data, pc.ctypes.data,
                                    eye.ctypes.data, _data(psh), _data(raster))
        if trial_data:
            return tr, nc, pc, eye, split_trial_data(psh, raster, self.num, proto)
        return tr, nc, pc, eye

    def run_protocol_step_rates(self, proto, step_rates, nsteps):
        """The eyelid driver with the MF rates of step s from row s % rows of
        step_rates [rows, numMF] (cbm_oracle_run_protocol_step_rates)."""
        lib = self.lib()
        p = ProtocolStruct.from_dict(proto)
        sizes = [ctypes.c_uint64() for _ in range(3)]
        lib.cbm_oracle_protocol_sizes(self.h, ctypes.byref(p), *[ctypes.byref(x) for x in sizes])
        nc = np.zeros(sizes[0].value, dtype=np.uint32)
        pc = np.zeros(sizes[1].value, dtype=np.uint32)
        eye = np.zeros(sizes[2].value, dtype=np.float32)
        rates = np.ascontiguousarray(step_rates, dtype=np.float32)
        lib.cbm_oracle_run_protocol_step_rates(self.h, ctypes.byref(p), rates.ctypes.data, rates.shape[0], nsteps,
                                               None, nc.ctypes.data, pc.ctypes.data, eye.ctypes.data)

    def save(self, path):
        if self.lib().cbm_oracle_save(self.h, os.fsencode(path)) != 0:
            raise RuntimeError("oracle save failed")


def _data(a):
    return None if a is None else a.ctypes.data


# the trial-data records in their order (cbm_oracle_trial_data_sizes)
TRIAL_PSH = [("go", "GO"), ("grInputGO", "GO"), ("goInputGO", "GO"), ("goOutSynScale", "GO"), ("mf", "MF"),
             ("sc", "SC"), ("bc", "BC"), ("pc", "PC"), ("io", "IO")]
TRIAL_RASTER = [("go", "GO"), ("sc", "SC"), ("bc", "BC"), ("pc", "PC"), ("nc", "NC"), ("io", "IO")]


def split_trial_data(psh, raster, num, proto):
    """{"psh": {name: f32 [bins][cells]}, "raster": {name: u32 [trials][rows][cells]}}
    from the concatenated records."""
    rec_from = proto["csOn"] - proto["preCS"]
    rec_len = proto["csOff"] + proto["postCS"] - rec_from
    bins = (rec_len + proto["binSteps"] - 1) // proto["binSteps"]
    rows, nd = rec_len // 32, proto["numDataTrials"]
    out = {"psh": {}, "raster": {}}
    off = 0
    for name, cell in TRIAL_PSH:
        n = bins * num[cell]
        out["psh"][name] = psh[off: off + n].reshape(bins, num[cell])
        off += n
    assert off == psh.size
    off = 0
    for name, cell in TRIAL_RASTER:
        n = nd * rows * num[cell]
        out["raster"][name] = raster[off: off + n].reshape(nd, rows, num[cell])
        off += n
    assert off == raster.size
    return out


PROTOCOL_FIELDS = [("trialSteps", "u"), ("csOn", "i"), ("csOff", "i"), ("csPhasicOff", "i"), ("csStartTrial", "u"),
                   ("plastOnDelay", "i"), ("plastOffDelay", "i"), ("plastLTD", "f"), ("plastLTP", "f"),
                   ("usErrDrive", "f"), ("mfSeed", "i"), ("mfThreshDecayTau", "f"), ("dataStartTrial", "u"),
                   ("numDataTrials", "u"), ("preCS", "i"), ("postCS", "i"), ("binSteps", "u"),
                   ("eyeGDecayTau", "f"), ("eyeGInc", "f"), ("eyeGShift", "f"), ("eyeGLeakRaw", "f"),
                   ("eyeMaxAmp", "f")]


class ProtocolStruct(ctypes.Structure):
    """cbm_oracle_protocol (oracle/cbm_oracle.h)."""
    _fields_ = [(n, {"u": ctypes.c_uint32, "i": ctypes.c_int32, "f": ctypes.c_float}[k]) for n, k in PROTOCOL_FIELDS]

    @classmethod
    def from_dict(cls, d):
        return cls(**{n: d[n] for n, _ in PROTOCOL_FIELDS})


def short_protocol(**kw):
    """A small eyelid protocol for tests: 400-step trials, CS 120-260."""
    p = dict(trialSteps=400, csOn=120, csOff=260, csPhasicOff=150, csStartTrial=1, plastOnDelay=40,
             plastOffDelay=30, plastLTD=-0.004, plastLTP=0.002, usErrDrive=1.0, mfSeed=11, mfThreshDecayTau=4.0,
             dataStartTrial=0, numDataTrials=3, preCS=60, postCS=80, binSteps=10, eyeGDecayTau=10.5,
             eyeGInc=0.012, eyeGShift=-0.13, eyeGLeakRaw=0.13, eyeMaxAmp=100.0)
    p.update(kw)
    return p


def statevar_protocol(mf_seed, tau=4.0):
    """The eyelid-driver fields a device state-variable input runs with
    (cbm_sim_set_statevar_input): no CS trial, no US, no plasticity window,
    no kept trial; the MF generator's seed and time constant."""
    return dict(trialSteps=1 << 30, csOn=0, csOff=0, csPhasicOff=0, csStartTrial=0xFFFFFFFF, plastOnDelay=0,
                plastOffDelay=0, plastLTD=0.0, plastLTP=0.0, usErrDrive=0.0, mfSeed=mf_seed, mfThreshDecayTau=tau,
                dataStartTrial=0, numDataTrials=0, preCS=0, postCS=1, binSteps=1, eyeGDecayTau=10.5, eyeGInc=0.012,
                eyeGShift=-0.13, eyeGLeakRaw=0.13, eyeMaxAmp=100.0)


def protocol_rates(num_mf, seed=0):
    """[3, num_mf] Hz: background 1-30, CS tonic and phasic raised on a random 10%."""
    rng = np.random.Generator(np.random.PCG64(seed + 500))
    bg = rng.uniform(1.0, 30.0, num_mf).astype(np.float32)
    tonic, phasic = bg.copy(), bg.copy()
    cs = rng.permutation(num_mf)[: max(1, num_mf // 10)]
    tonic[cs] = 80.0
    phasic[cs] = 150.0
    return np.stack([bg, tonic, phasic])


def ref_run_protocol(state_path, proto, rates, nsteps, seeds, mf_population=None, data_file=None,
                     session_file=None):
    """oracle/_ref/ref_run in protocol mode: (trace bytes, records bytes).
    With mf_population (a path), the reference's ECMFPopulation estimated
    from the run's ECTrialsData is written there; with data_file, the
    ECTrialsData itself (writeData); with session_file, the final state and
    the ECTrialsData as the driver's writeDataToFile writes them."""
    with tempfile.TemporaryDirectory() as d:
        rp = os.path.join(d, "rates.f32")
        np.ascontiguousarray(rates, dtype=np.float32).tofile(rp)
        pp = os.path.join(d, "protocol.txt")
        with open(pp, "w") as f:
            for n, _ in PROTOCOL_FIELDS:
                f.write(f"{n} {proto[n]!r}\n")
            f.write(f"rates {rp}\n")
        trp, rec = os.path.join(d, "trace.bin"), os.path.join(d, "records.bin")
        cmd = [REF_RUN, state_path, "-", str(nsteps), trp, "-"] + [str(s) for s in seeds] + ["-p", pp, "-r", rec]
        if mf_population:
            cmd += ["-m", mf_population]
        if data_file:
            cmd += ["-d", data_file]
        if session_file:
            cmd += ["-s", session_file]
        subprocess.run(cmd, check=True, capture_output=True)
        return np.fromfile(trp, dtype=np.uint8), np.fromfile(rec, dtype=np.uint8)


def split_ref_records(rec, num, proto):
    """The RECORDS file of ref_run -p as a dict: nc, pc (u32 per trial),
    eye, gr (f32 [bins][numGR]), psh {name: f32 [bins][cells]} (the driver's
    ECTrialsData histograms; "gr" covers numGR / 10 cells there), raster
    {name: u32 [trials][rows][cells]}, eyelid_out (the driver's smoothed
    eyelid trace, f32 [trials][window])."""
    rec_from = proto["csOn"] - proto["preCS"]
    rec_len = proto["csOff"] + proto["postCS"] - rec_from
    bins = (rec_len + proto["binSteps"] - 1) // proto["binSteps"]
    nd, rows = proto["numDataTrials"], rec_len // 32
    out, off = {"psh": {}, "raster": {}}, 0

    def take(n, dtype):
        nonlocal off
        a = rec[off: off + 4 * n].view(dtype)
        off += 4 * n
        return a

    out["nc"] = take(nd * bins * num["NC"], np.uint32)
    out["pc"] = take(nd * bins * num["PC"], np.uint32)
    out["eye"] = take(nd * rec_len, np.float32)
    out["gr"] = take(bins * num["GR"], np.float32).reshape(bins, num["GR"])
    for name, cell in TRIAL_PSH + [("gr", None)]:
        n = num[cell] if cell else num["GR"] // 10
        out["psh"][name] = take(bins * n, np.float32).reshape(bins, n)
    for name, cell in TRIAL_RASTER:
        out["raster"][name] = take(nd * rows * num[cell], np.uint32).reshape(nd, rows, num[cell])
    out["eyelid_out"] = take(nd * rec_len, np.float32).reshape(nd, rec_len)
    assert off == rec.size
    return out


def raster_rows_filled(proto):
    """Rows of the trial-data rasters that a run of whole trials fills, in
    (trial, row) order: one per 32nd window step after the first, so
    (recLen - 1) // 32 per trial against recLen // 32 rows a raster trial."""
    rec_len = proto["csOff"] + proto["postCS"] - (proto["csOn"] - proto["preCS"])
    nd, rows = proto["numDataTrials"], rec_len // 32
    return min(nd * rows, nd * ((rec_len - 1) // 32))


def gr_psh_from_trace(trace, proto, n_gr):
    """GR peri-stimulus histogram [bins][numGR] of a protocol run from its
    per-step trace records (protocol started at step 0): in the recording
    window of every kept trial, each GR spike adds one to its bin, all kept
    trials into one histogram (the eyelid driver's updatePSH("gr"))."""
    rec_from = proto["csOn"] - proto["preCS"]
    rec_len = proto["csOff"] + proto["postCS"] - rec_from
    bins = (rec_len + proto["binSteps"] - 1) // proto["binSteps"]
    out = np.zeros((bins, n_gr), np.uint32)
    nb = (n_gr + 7) // 8
    first, last = proto["dataStartTrial"], proto["dataStartTrial"] + proto["numDataTrials"]
    for s in range(trace.shape[0]):
        time, trial = s % proto["trialSteps"], s // proto["trialSteps"]
        ct = time - rec_from
        if first <= trial < last and 0 <= ct < rec_len:
            out[ct // proto["binSteps"]] += np.unpackbits(np.asarray(trace[s][:nb], np.uint8), bitorder="little")[:n_gr]
    return out


def events_file(events, path):
    with open(path, "w") as f:
        for t in sorted(events):
            for ev in events[t]:
                f.write(f"{t} {ev[0]} " + " ".join(str(x) for x in ev[1:]) + "\n")


def ref_available():
    return os.path.exists(REF_RUN)


def ref_run(state_path, mf, seeds, events=None, num_gpus=1, final_path=None):
    """The reference's own host code (oracle/_ref/ref_run) on the same input."""
    mf = np.ascontiguousarray(mf, dtype=np.uint8)
    with tempfile.TemporaryDirectory() as d:
        mfp = os.path.join(d, "mf.u8")
        mf.tofile(mfp)
        trp = os.path.join(d, "trace.bin")
        cmd = [REF_RUN, state_path, mfp, str(mf.shape[0]), trp, final_path or "-"] + [str(s) for s in seeds]
        if events:
            evp = os.path.join(d, "ev.txt")
            events_file(events, evp)
            cmd += ["-e", evp]
        env = dict(os.environ)
        if num_gpus > 1:
            env["CBM_FAKE_NUM_GPUS"] = str(num_gpus)
            cmd += ["-g", str(int(np.log2(num_gpus)))]
        subprocess.run(cmd, check=True, capture_output=True, env=env)
        return np.fromfile(trp, dtype=np.uint8)


def product_record(sim, num):
    """One trace record of a CBMSimCore in the oracle's layout."""
    inet = sim.getInputNet()
    parts = [np.packbits(inet.exportAPGR().astype(bool), bitorder="little"), inet.exportAPGO(),
             inet.exportVmGO().view(np.uint8), inet.exportSumGRInputGO().view(np.uint8),
             inet.exportAPSC(), inet.exportVmSC().view(np.uint8)]
    for z in sim.getMZoneList():
        parts += [z.exportAPBC(), z.exportVmBC().view(np.uint8), z.exportAPPC(), z.exportVmPC().view(np.uint8),
                  z.exportAPIO(), z.exportVmIO().view(np.uint8), z.exportAPNC(), z.exportVmNC().view(np.uint8)]
    return np.concatenate([np.asarray(p, dtype=np.uint8).ravel() for p in parts])


def product_run(sim, mf, events=None, t0=0, record=True):
    recs = []
    zones = sim.getMZoneList()
    inet = sim.getInputNet()
    for s in range(mf.shape[0]):
        for ev in (events or {}).get(t0 + s + 1, []):
            k = ev[0]
            if k == "errdrive":
                sim.updateErrDrive(ev[1], ev[2])
            elif k == "plast":
                zones[ev[1]].setGRPCPlastSteps(ev[2], ev[3])
            elif k == "plastreset":
                zones[ev[1]].resetGRPCPlastSteps()
            elif k == "grgoinc":
                inet.setGIncGRtoGO(ev[1])
            elif k == "grgoincreset":
                inet.resetGIncGRtoGO()
        sim.updateMFInput(mf[s])
        sim.calcActivity()
        if record:
            recs.append(product_record(sim, None))
    return np.stack(recs) if record else None


def record_layout(num):
    """(name, dtype, count) of the fields of one trace record."""
    lay = [("apGR", np.uint8, (num["GR"] + 7) // 8), ("apGO", np.uint8, num["GO"]), ("vGO", np.float32, num["GO"]),
           ("sumGRInputGO", np.uint32, num["GO"]), ("apSC", np.uint8, num["SC"]), ("vSC", np.float32, num["SC"])]
    for z in range(num["zones"]):
        lay += [(f"apBC{z}", np.uint8, num["BC"]), (f"vBC{z}", np.float32, num["BC"]),
                (f"apPC{z}", np.uint8, num["PC"]), (f"vPC{z}", np.float32, num["PC"]),
                (f"apIO{z}", np.uint8, num["IO"]), (f"vIO{z}", np.float32, num["IO"]),
                (f"apNC{z}", np.uint8, num["NC"]), (f"vNC{z}", np.float32, num["NC"])]
    return lay


def same_values(x, y):
    """Bitwise equality, except that any two NaNs are equal: the host CPU and
    the GPU encode the NaN of an invalid operation with different sign and
    payload bits, which carry no meaning."""
    x, y = np.asarray(x), np.asarray(y)
    if x.dtype.kind == "f":
        return (x.view(np.uint8).reshape(x.size, -1) == y.view(np.uint8).reshape(y.size, -1)).all(axis=1) | \
            (np.isnan(x) & np.isnan(y))
    return x == y


def first_difference(a, b, num):
    """Human-readable location of the first differing value of two traces."""
    rb = a.shape[-1]
    a = a.reshape(-1, rb)
    b = b.reshape(a.shape)
    cand = np.nonzero((a != b).any(axis=1))[0]
    for step in cand:
        off = 0
        for name, dt, cnt in record_layout(num):
            nb = np.dtype(dt).itemsize * cnt
            x = a[step, off:off + nb].view(dt)
            y = b[step, off:off + nb].view(dt)
            if not same_values(x, y).all():
                return f"step {int(step) + 1}: field {name}"
            off += nb
    return None


def counter_mf(num_mf, steps, seed, rate_lo=0.001, rate_hi=0.06):
    """Deterministic MF spikes from the counter-based stream: fibre i fires at
    step s with a fixed per-fibre probability in [rate_lo, rate_hi)."""
    from cerebellum_simulation_b200.networks import uniform24
    rates = rate_lo + (rate_hi - rate_lo) * uniform24(seed, 0x52415445, np.arange(num_mf, dtype=np.uint64))
    out = np.empty((steps, num_mf), dtype=np.uint8)
    for s in range(steps):
        u = uniform24(seed, 0x4D46494E, (np.uint64(s + 1) << np.uint64(20)) | np.arange(num_mf, dtype=np.uint64))
        out[s] = u < rates
    return out


def sha(b):
    return hashlib.sha256(np.ascontiguousarray(b).tobytes()).hexdigest()


def golden_state(name, dest_dir):
    """Decompress tests/golden/<name>.state.xz into dest_dir; returns the path."""
    out = os.path.join(dest_dir, name + ".state")
    with lzma.open(os.path.join(GOLDEN, name + ".state.xz")) as f, open(out, "wb") as g:
        g.write(f.read())
    return out


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def golden_large_case(name):
    """(network, MF input [steps, numMF], events) of a large golden fixture
    (tests/golden/make_golden.py records the reference's run of it).

    config2: the 1M-GR network over 1000 steps of eyelid-coded MF input with
    a CS from 50 to 250, large LTD/LTP steps from step 2 and an error drive at
    249 and 749; GR history bit 39, which gates PF->PC plasticity
    (kernels.cu:282-291), is first set about 200 steps in, so weights move in
    the last 800 steps.  config3: the dense 4M-GR network over 400 steps of
    state-variable-coded input, with plasticity from step 1 and an error drive
    at 40 and 340."""
    from cerebellum_simulation_b200 import networks
    if name == "config2":
        steps = 1000
        return (networks.config2_network(seed=0),
                networks.eyelid_mf_stream(1024, steps, seed=0, cs_on=50, cs_off=250),
                {2: [("plast", 0, -0.01, 0.005)], 249: [("errdrive", 0, 1.0)], 749: [("errdrive", 0, 1.0)]})
    if name == "config3":
        steps = 400
        return (networks.config3_network(seed=0), networks.config3_mf_stream(1024, steps, seed=0),
                {1: [("plast", 0, -0.0005, 0.0005)], 40: [("errdrive", 0, 1.0)], 340: [("errdrive", 0, 1.0)]})
    raise KeyError(name)


def state_array_digests(path):
    """SHA-256 of every array of a state file, by (zone, name): lets a run
    whose few FP-tolerant arrays may differ in the last bits be compared
    array by array with a recorded one."""
    import cerebellum_simulation_b200 as cbm
    from test_gpu_parity import INNET_ACT, INNET_CON, ZONE_ACT
    st = cbm.CBMState(path)
    out = {}
    for n in INNET_CON + INNET_ACT:
        out[f"-1/{n}"] = sha(st.array(n, -1))
    for z in range(st.getNumZones()):
        for n in ZONE_ACT:
            out[f"{z}/{n}"] = sha(st.array(n, z))
    return out


# The GO glutamate/mGluR state uses the double-precision exp of the host C
# library in the reference and CUDA's double exp on the device; the two can
# differ in the last double bit, which reaches these float arrays as at most a
# few float ulps.  No spike depends on them (innet.cpp:850-858).
FP_TOLERANT_ARRAYS = {"gluGO", "mGluRGO", "gMGluRIncGO", "gMGluRGO"}
FP_RTOL = 1e-5


def build_facade_check(dest_dir):
    """Compile tests/cpp/facade_check.cpp against include/cbm_core.hpp and
    libcbm_b200.so; returns the executable's path."""
    import subprocess
    import cerebellum_simulation_b200 as cbm
    libdir = os.path.dirname(cbm.LIB_PATH)
    exe = os.path.join(dest_dir, "facade_check")
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "facade_check.cpp"), "-L", libdir, "-lcbm_b200",
           f"-Wl,-rpath,{libdir}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe
