"""B200-native cerebellar network step behind the reference's CBM_CORE_LIB API.

Python mirror of the reference's host interface (``CBMState``,
``CBMSimCore``, ``InNetInterface``, ``MZoneInterface``; see
``include/cbm_b200.h`` for the C ABI and the reference lines each call
replaces).  All computation runs in ``libcbm_b200.so`` on the GPU; importing
this package fails if the library has not been built.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libcbm_b200.so")

CBM_OK = 0
_DTYPES = {0: np.uint8, 1: np.int32, 2: np.uint32, 3: np.float32, 4: np.uint64}

# enum cbm_field
FIELDS = [
    "AP_GR", "VM_GR", "GESUM_GR", "GISUM_GR", "APBUF_GR", "HIST_GR", "THRESH_GR", "GKCA_GR",
    "AP_GO", "VM_GO", "APBUF_GO", "SUM_GR_INPUT_GO", "SUM_GO_INPUT_GO", "GO_OUT_SCALE_GOGO",
    "AP_SC", "VM_SC", "APBUF_SC", "HIST_MF", "APBUF_MF",
    "AP_BC", "VM_BC", "APBUF_BC", "AP_PC", "VM_PC", "APBUF_PC", "AP_IO", "VM_IO", "APBUF_IO",
    "AP_NC", "VM_NC", "APBUF_NC", "PFPC_WEIGHT", "MFNC_WEIGHT",
]
FIELD = {n: i for i, n in enumerate(FIELDS)}
_FIELD_DTYPE = {
    "AP": np.uint8, "VM": np.float32, "GESUM": np.float32, "GISUM": np.float32, "APBUF": np.uint32,
    "HIST": np.uint64, "THRESH": np.float32, "GKCA": np.float32, "SUM": None, "GO": np.float32,
    "PFPC": np.float32, "MFNC": np.float32,
}


def _field_dtype(name):
    if name == "SUM_GR_INPUT_GO":
        return np.uint32
    if name in ("SUM_GO_INPUT_GO", "GO_OUT_SCALE_GOGO"):
        return np.float32
    if name == "HIST_MF":
        return np.uint8
    return _FIELD_DTYPE[name.split("_")[0]]


# ECTrialsData record kinds (CBM_REC_PSH_*, CBM_REC_RASTER_*) and the cells
# each covers, under the eyelid driver's names
TRIAL_PSH = {"go": (4, "numGO"), "grInputGO": (5, "numGO"), "goInputGO": (6, "numGO"),
             "goOutSynScale": (7, "numGO"), "mf": (8, "numMF"), "sc": (9, "numSC"), "bc": (10, "numBC"),
             "pc": (11, "numPC"), "io": (12, "numIO")}
TRIAL_RASTER = {"go": (13, "numGO"), "sc": (14, "numSC"), "bc": (15, "numBC"), "pc": (16, "numPC"),
                "nc": (17, "numNC"), "io": (18, "numIO")}


def eyelid_out(raw, num_ts_smooth=4):
    """The eyelid driver's recorded eyelid trace (EyelidOut::updateData,
    CBM_DATA_LIB_DEV/src/outdata/eyelidout.cpp) from the integrator's raw
    output [trials, window steps]: the first num_ts_smooth - 1 values as
    they are, then each value the float mean of the previous num_ts_smooth -
    1 recorded (already smoothed) values and the new one, summed in order."""
    raw = np.atleast_2d(np.asarray(raw, dtype=np.float32))
    out = np.zeros_like(raw)
    n = int(num_ts_smooth)
    for ts in range(raw.shape[1]):
        if ts < n - 1:
            out[:, ts] = raw[:, ts]
            continue
        avg = np.zeros(raw.shape[0], np.float32)
        for j in range(-(n - 1), 0):
            avg = (avg + out[:, ts + j]).astype(np.float32)
        avg = (avg + raw[:, ts]).astype(np.float32)
        out[:, ts] = (avg / np.float32(n)).astype(np.float32)
    return out


class CBMError(RuntimeError):
    """A failed call of the C ABI; .code holds the CBM_ERR_* status."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python cerebellum_simulation_b200/build.py`")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, U, F, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint, ctypes.c_float, ctypes.c_double, ctypes.c_char_p
    U64, U32 = ctypes.c_uint64, ctypes.c_uint32
    sig = {
        "cbm_last_error": (S, []),
        "cbm_state_load": (I, [S, ctypes.POINTER(P)]),
        "cbm_state_new": (I, [S, S, U, P, ctypes.POINTER(P)]),
        "cbm_state_save": (I, [P, S]),
        "cbm_state_generate": (I, [S, S, U, P, ctypes.POINTER(P)]),
        "cbm_state_load_mem": (I, [P, U64, ctypes.POINTER(U64), ctypes.POINTER(P)]),
        "cbm_state_save_mem": (I, [P, P, U64, ctypes.POINTER(U64)]),
        "cbm_sim_save_mem": (I, [P, P, U64, ctypes.POINTER(U64)]),
        "cbm_state_free": (None, [P]),
        "cbm_state_num_zones": (I, [P, ctypes.POINTER(U)]),
        "cbm_state_array": (I, [P, S, I, ctypes.POINTER(P), ctypes.POINTER(U64), ctypes.POINTER(I)]),
        "cbm_state_con_param": (I, [P, S, ctypes.POINTER(U32)]),
        "cbm_state_act_param": (I, [P, S, ctypes.POINTER(D)]),
        "cbm_state_set_act_param": (I, [P, S, F]),
        "cbm_sim_create": (I, [P, P, I, ctypes.POINTER(P)]),
        "cbm_sim_create_resident": (I, [P, P, I, U64, ctypes.POINTER(P)]),
        "cbm_sim_update_mf": (I, [P, P]),
        "cbm_sim_calc_activity": (I, [P]),
        "cbm_sim_update_err_drive": (I, [P, U, F]),
        "cbm_sim_set_plast_steps": (I, [P, U, F, F]),
        "cbm_sim_reset_plast_steps": (I, [P, U]),
        "cbm_sim_set_ginc_grgo": (I, [P, F]),
        "cbm_sim_reset_ginc_grgo": (I, [P]),
        "cbm_sim_export": (I, [P, I, U, P, U64]),
        "cbm_sim_field_bytes": (U64, [P, I]),
        "cbm_sim_write_to_state": (I, [P]),
        "cbm_sim_save": (I, [P, S]),
        "cbm_sim_steps_done": (I, [P, ctypes.POINTER(U64)]),
        "cbm_sim_mf_words": (I, [P, ctypes.POINTER(U32)]),
        "cbm_sim_load_mf_stream": (I, [P, P, U64]),
        "cbm_sim_run": (I, [P, U64, U32, ctypes.POINTER(F), ctypes.POINTER(F)]),
        "cbm_sim_algorithmic_bytes_per_step": (D, [P]),
        "cbm_sim_layout_bytes_per_step": (D, [P]),
        "cbm_sim_pass_geometry": (I, [P, ctypes.POINTER(U32), ctypes.POINTER(U32), ctypes.POINTER(U32),
                                      ctypes.POINTER(U32)]),
        "cbm_sim_timer_start": (I, [P]),
        "cbm_sim_last_tail_ms": (I, [P, ctypes.POINTER(F)]),
        "cbm_sim_run_flushed": (I, [P, U64, U64, ctypes.POINTER(F)]),
        "cbm_sim_run_flushed_kernels": (I, [P, U64, U64, ctypes.POINTER(F), ctypes.POINTER(F)]),
        "cbm_sim_set_eyelid_protocol": (I, [P, P]),
        "cbm_batch_create": (I, [P, U32, P, I, P]),
        "cbm_batch_destroy": (None, [P]),
        "cbm_batch_set_eyelid_protocol": (I, [P, U32, P]),
        "cbm_batch_run": (I, [P, U64, U32, ctypes.POINTER(F)]),
        "cbm_batch_autotune": (I, [P, U32, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(F)]),
        "cbm_batch_pass_geometry": (I, [P, ctypes.POINTER(U32), ctypes.POINTER(U32), ctypes.POINTER(U32),
                                        ctypes.POINTER(U32)]),
        "cbm_batch_trial_record_bytes": (U64, [P, U32, I]),
        "cbm_batch_trial_record": (I, [P, U32, I, P, U64]),
        "cbm_batch_write_to_state": (I, [P, U32]),
        "cbm_batch_num_gr": (U64, [P]),
        "cbm_sim_trial_record_bytes": (U64, [P, I]),
        "cbm_sim_trial_record": (I, [P, I, P, U64]),
        "cbm_sim_record_gr": (I, [P]),
        "cbm_state_param_names": (I, [P, I, ctypes.c_char_p, U64, ctypes.POINTER(U64)]),
        "cbm_state_raw_param": (I, [P, I, ctypes.c_char_p, ctypes.POINTER(D)]),
        "cbm_sim_record_trial_data": (I, [P]),
        "cbm_sim_timer_stop": (I, [P, ctypes.POINTER(F)]),
        "cbm_sim_destroy": (None, [P]),
        "cbm_device_expf": (I, [I, P, P, U64]),
        "cbm_device_exp": (I, [I, P, P, U64]),
        "cbm_sim_set_statevar_input": (I, [P, P]),
        "cbm_batch_record_trial_data": (I, [P, U]),
        "cbm_sim_statevar_rates": (I, [P, U64, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _check(rc):
    if rc != CBM_OK:
        raise CBMError(rc, lib.cbm_last_error().decode())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _serialised(save):
    """Bytes of one of the C ABI's two-call serialisations (size, then data)."""
    n = ctypes.c_uint64()
    _check(save(None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value)
    _check(save(buf, n.value, ctypes.byref(n)))
    return buf.raw[: n.value]


class CBMState:
    """The reference's CBMState (CBM_STATE_LIB_DEV/CBMStateInclude/interfaces/cbmstate.h:37-62)."""

    def __init__(self, path=None, _handle=None):
        """CBMState(fstream&): path is a state file's name, or a binary file
        object positioned at a state, which is left positioned just after it
        (where the eyelid driver's session file continues with its trial
        data)."""
        self._h = ctypes.c_void_p()
        if _handle is not None:
            self._h = _handle
        elif hasattr(path, "read"):
            start = path.tell()
            data = path.read()
            used = ctypes.c_uint64()
            _check(lib.cbm_state_load_mem(data, len(data), ctypes.byref(used), ctypes.byref(self._h)))
            path.seek(start + used.value)
        elif path is not None:
            _check(lib.cbm_state_load(os.fsencode(path), ctypes.byref(self._h)))
        else:
            raise ValueError("CBMState needs a state file path (or use CBMState.new)")

    @classmethod
    def generate(cls, con_text, act_text, n_zones=1, innet_seed=None, zone_con_seeds=None, zone_act_seeds=None):
        """CBMState(actPF, conPF, nZones, innetCRSeed, mzoneCRSeed,
        mzoneARSeed): the network with the reference's own generator and
        random sequence (cbm_state_generate); without seeds they are drawn
        from the wall clock, as CBMState(actPF, conPF, nZones) does."""
        h = ctypes.c_void_p()
        seeds = None
        if innet_seed is not None:
            zc = list(zone_con_seeds) if zone_con_seeds is not None else [innet_seed + 1 + z for z in range(n_zones)]
            za = list(zone_act_seeds) if zone_act_seeds is not None else [0] * n_zones
            seeds = np.asarray([innet_seed] + zc[:n_zones] + za[:n_zones], dtype=np.int32)
        _check(lib.cbm_state_generate(con_text.encode(), act_text.encode(), n_zones, _ptr(seeds), ctypes.byref(h)))
        return cls(_handle=h)

    @classmethod
    def new(cls, con_text, act_text, n_zones=1, wiring_seeds=None):
        """CBMState(actPF, conPF, nZones, ...) with input-net wiring left to the caller."""
        h = ctypes.c_void_p()
        seeds = None if wiring_seeds is None else np.asarray(wiring_seeds, dtype=np.int32)
        _check(lib.cbm_state_new(con_text.encode(), act_text.encode(), n_zones, _ptr(seeds), ctypes.byref(h)))
        return cls(_handle=h)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and not getattr(self, "_borrowed", False):
            lib.cbm_state_free(self._h)
            self._h = ctypes.c_void_p()

    def writeState(self, path):
        """writeState(fstream&): to a file name, or into a binary file object
        at its position."""
        if hasattr(path, "write"):
            path.write(_serialised(lambda d, c, n: lib.cbm_state_save_mem(self._h, d, c, n)))
        else:
            _check(lib.cbm_state_save(self._h, os.fsencode(path)))

    def getNumZones(self):
        n = ctypes.c_uint()
        _check(lib.cbm_state_num_zones(self._h, ctypes.byref(n)))
        return n.value

    def array(self, name, zone=-1):
        """numpy view of a state array; writes go straight into the state."""
        data, count, dt = ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_int()
        _check(lib.cbm_state_array(self._h, name.encode(), zone, ctypes.byref(data), ctypes.byref(count),
                                   ctypes.byref(dt)))
        dtype = np.dtype(_DTYPES[dt.value])
        if count.value == 0:
            return np.zeros(0, dtype=dtype)
        buf = (ctypes.c_char * (count.value * dtype.itemsize)).from_address(data.value)
        buf._owner = self  # the view keeps the state (and its memory) alive
        return np.frombuffer(buf, dtype=dtype)

    def con(self, name):
        v = ctypes.c_uint32()
        _check(lib.cbm_state_con_param(self._h, name.encode(), ctypes.byref(v)))
        return v.value

    def act(self, name):
        v = ctypes.c_double()
        _check(lib.cbm_state_act_param(self._h, name.encode(), ctypes.byref(v)))
        return v.value

    def setActParam(self, key, value):
        _check(lib.cbm_state_set_act_param(self._h, key.encode(), value))

    # the reference's accessor interfaces (cbmstate.cpp:105-146)
    def getConnectivityParams(self):
        return IConnectivityParams(self)

    def getActivityParams(self):
        return IActivityParams(self)

    def getInnetConState(self):
        return IInNetConState(self)

    def getMZoneActState(self, zoneN):
        if not 0 <= zoneN < self.getNumZones():
            raise CBMError(1, "zone out of range")
        return IMZoneActState(self, zoneN)

    def equivalent(self, other):
        """CBMState::equivalent (cbmstate.cpp:105-121,
        innetconnectivitystate.cpp:228-243): zone count, MF->GL glomeruli and
        the GO->GR / GR<-GO counts."""
        return self.getNumZones() == other.getNumZones() and all(
            np.array_equal(self.array(n), other.array(n))
            for n in ("haspGLfromMFtoGL", "numpGOfromGOtoGR", "numpGRfromGOtoGR"))

    def _param_names(self, which):
        need = ctypes.c_uint64()
        lib.cbm_state_param_names(self._h, which, None, 0, ctypes.byref(need))
        buf = ctypes.create_string_buffer(need.value)
        _check(lib.cbm_state_param_names(self._h, which, buf, need.value, ctypes.byref(need)))
        return buf.value.decode().split()

    def _raw_param(self, which, name):
        v = ctypes.c_double()
        rc = lib.cbm_state_raw_param(self._h, which, name.encode(), ctypes.byref(v))
        return v.value if rc == CBM_OK else None


class IConnectivityParams:
    """IConnectivityParams (CBM_STATE_LIB_DEV/CBMStateInclude/interfaces/iconnectivityparams.h)."""

    def __init__(self, state):
        self._s = state

    def getParamCopy(self):
        return {n: int(self._s._raw_param(0, n)) for n in self._s._param_names(0)}

    def showParams(self, out=None):
        """The parameter file's keys and values in key order."""
        import sys
        for k, v in self.getParamCopy().items():
            print(k, v, file=out or sys.stdout)


for _name, _field in (("getGOX", "goX"), ("getGOY", "goY"), ("getGRX", "grX"), ("getGRY", "grY"),
                      ("getGLX", "glX"), ("getGLY", "glY"), ("getNumMF", "numMF"), ("getNumGO", "numGO"),
                      ("getNumGR", "numGR"), ("getNumGL", "numGL"), ("getNumSC", "numSC"), ("getNumBC", "numBC"),
                      ("getNumPC", "numPC"), ("getNumNC", "numNC"), ("getNumIO", "numIO")):
    setattr(IConnectivityParams, _name, (lambda f: lambda self: self._s.con(f))(_field))


class IActivityParams:
    """IActivityParams (iactivityparams.h): getParam / setParam work on the
    parameter file's keys; setParam re-derives the step's values
    (activityparams.cpp:418-434)."""

    def __init__(self, state):
        self._s = state

    def getMSPerTimeStep(self):
        return int(self._s.act("msPerTimeStep"))

    def getParamCopy(self):
        return {n: float(np.float32(self._s._raw_param(1, n))) for n in self._s._param_names(1)}

    def getParam(self, paramName):
        v = self._s._raw_param(1, paramName)
        return 0.0 if v is None else float(np.float32(v))  # an unknown key reads 0, as paramMap[key] does

    def setParam(self, paramName, value):
        return lib.cbm_state_set_act_param(self._s._h, paramName.encode(), value) == CBM_OK

    def showParams(self, out=None):
        import sys
        for k, v in self.getParamCopy().items():
            print(k, v, file=out or sys.stdout)


class IInNetConState:
    """IInNetConState (iinnetconstate.h): per-cell connection lists of the
    input network, read from and (GO->GO pairs) edited in the state arrays
    (innetconnectivitystate.cpp:245-470)."""

    _LISTS = {"getpGOfromGOtoGLCon": "GOfromGOtoGL", "getpGOfromGLtoGOCon": "GOfromGLtoGO",
              "getpMFfromMFtoGLCon": "MFfromMFtoGL", "getpGLfromGLtoGRCon": "GLfromGLtoGR",
              "getpGRfromMFtoGR": "GRfromMFtoGR", "getpGRfromGOtoGR": "GRfromGOtoGR",
              "getpGOfromGRtoGOCon": "GOfromGRtoGO", "getpGOfromGOtoGRCon": "GOfromGOtoGR",
              "getpMFfromMFtoGRCon": "MFfromMFtoGR", "getpMFfromMFtoGOCon": "MFfromMFtoGO",
              "getpGOfromMFtoGOCon": "GOfromMFtoGO", "getpGOOutGOGOCon": "GOGABAOutGOGO",
              "getpGOInGOGOCon": "GOGABAInGOGO"}

    def __init__(self, state):
        self._s = state

    def _table(self, key):
        num, p = self._s.array("nump" + key), self._s.array("p" + key)
        return num, p.reshape(num.size, -1)

    def _con(self, key, n):
        num, p = self._table(key)
        return [int(x) for x in p[n, : num[n]]]

    def __getattr__(self, name):
        if name in IInNetConState._LISTS:
            return lambda n: self._con(IInNetConState._LISTS[name], n)
        raise AttributeError(name)

    def getpGRPopfromMFtoGR(self):
        return [self._con("GRfromMFtoGR", i) for i in range(self._s.con("numGR"))]

    def getpGRPopfromGOtoGR(self):
        return [self._con("GRfromGOtoGR", i) for i in range(self._s.con("numGR"))]

    def getpGOPopfromMFtoGOCon(self):
        return [self._con("GOfromMFtoGO", i) for i in range(self._s.con("numGO"))]

    def getGOIncompIndfromGRtoGO(self):
        return list(np.nonzero(self._s.array("numpGOfromGRtoGO") < self._s.con("maxnumpGOfromGRtoGO"))[0])

    def getGRIncompIndfromGRtoGO(self):
        return list(np.nonzero(self._s.array("numpGRfromGRtoGO") < self._s.con("maxnumpGRfromGRtoGO"))[0])

    def addGOGOConPair(self, srcGON, destGON):
        on, op = self._table("GOGABAOutGOGO")
        inn, ip = self._table("GOGABAInGOGO")
        if on[srcGON] >= op.shape[1] or inn[destGON] >= ip.shape[1]:
            return False
        op[srcGON, on[srcGON]] = destGON
        on[srcGON] += 1
        ip[destGON, inn[destGON]] = srcGON
        inn[destGON] += 1
        return True

    def deleteGOGOConPair(self, srcGON, destGON):
        on, op = self._table("GOGABAOutGOGO")
        inn, ip = self._table("GOGABAInGOGO")
        hit = np.nonzero(op[srcGON, : on[srcGON]] == destGON)[0]
        if hit.size == 0:
            return False
        k = on[srcGON]
        op[srcGON, hit[0]: k - 1] = op[srcGON, hit[0] + 1: k].copy()
        on[srcGON] -= 1
        hit = np.nonzero(ip[destGON, : inn[destGON]] == srcGON)[0]  # the last match, as the reference
        if hit.size:
            k = inn[destGON]
            ip[destGON, hit[-1]: k - 1] = ip[destGON, hit[-1] + 1: k].copy()
            inn[destGON] -= 1
        return True


class IMZoneActState:
    """IMZoneActState (imzoneactstate.h, mzoneactivitystate.cpp:202-228)."""

    def __init__(self, state, zone):
        self._s, self._z = state, zone

    def getGRPCSynWeightLinear(self):
        return self._s.array("pfSynWeightPC", self._z).copy()

    def resetGRPCSynWeight(self):
        self._s.array("pfSynWeightPC", self._z)[:] = np.float32(self._s.act("initSynWofGRtoPC"))


class _Exporter:
    def __init__(self, sim, zone):
        self._sim = sim
        self._zone = zone
        self._shapes = {}  # field -> (id, bytes, dtype, count); sizes are fixed per network

    def _export(self, field):
        sh = self._shapes.get(field)
        if sh is None:
            fid = FIELD[field]
            nbytes = lib.cbm_sim_field_bytes(self._sim._h, fid)
            dt = np.dtype(_field_dtype(field))
            sh = self._shapes[field] = (fid, nbytes, dt, nbytes // dt.itemsize)
        fid, nbytes, dt, count = sh
        out = np.empty(count, dtype=dt)
        _check(lib.cbm_sim_export(self._sim._h, fid, self._zone, out.ctypes.data, nbytes))
        return out


class InNet(_Exporter):
    """InNetInterface (CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/innetinterface.h:18-41)."""

    def setGIncGRtoGO(self, inc):
        _check(lib.cbm_sim_set_ginc_grgo(self._sim._h, inc))

    def resetGIncGRtoGO(self):
        _check(lib.cbm_sim_reset_ginc_grgo(self._sim._h))

    def exportAPSC(self): return self._export("AP_SC")
    def exportAPGO(self): return self._export("AP_GO")
    def exportAPGR(self): return self._export("AP_GR")
    def exportHistMF(self): return self._export("HIST_MF")
    def exportAPBufMF(self): return self._export("APBUF_MF")
    def exportAPBufGR(self): return self._export("APBUF_GR")
    def exportAPBufGO(self): return self._export("APBUF_GO")
    def exportAPBufSC(self): return self._export("APBUF_SC")
    def exportVmGR(self): return self._export("VM_GR")
    def exportVmGO(self): return self._export("VM_GO")
    def exportVmSC(self): return self._export("VM_SC")
    def exportGESumGR(self): return self._export("GESUM_GR")
    def exportGISumGR(self): return self._export("GISUM_GR")
    def exportSumGRInputGO(self): return self._export("SUM_GR_INPUT_GO")
    def exportSumGOInputGO(self): return self._export("SUM_GO_INPUT_GO")
    def exportGOOutSynScaleGOGO(self): return self._export("GO_OUT_SCALE_GOGO")
    def exportHistoryGR(self): return self._export("HIST_GR")


class MZone(_Exporter):
    """MZoneInterface (CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/mzoneinterface.h:18-34)."""

    def setGRPCPlastSteps(self, ltdStep, ltpStep):
        _check(lib.cbm_sim_set_plast_steps(self._sim._h, self._zone, ltdStep, ltpStep))

    def resetGRPCPlastSteps(self):
        _check(lib.cbm_sim_reset_plast_steps(self._sim._h, self._zone))

    def exportAPBC(self): return self._export("AP_BC")
    def exportAPPC(self): return self._export("AP_PC")
    def exportAPIO(self): return self._export("AP_IO")
    def exportAPNC(self): return self._export("AP_NC")
    def exportAPBufBC(self): return self._export("APBUF_BC")
    def exportAPBufPC(self): return self._export("APBUF_PC")
    def exportAPBufIO(self): return self._export("APBUF_IO")
    def exportAPBufNC(self): return self._export("APBUF_NC")
    def exportVmBC(self): return self._export("VM_BC")
    def exportVmPC(self): return self._export("VM_PC")
    def exportVmNC(self): return self._export("VM_NC")
    def exportVmIO(self): return self._export("VM_IO")
    def exportPFPCWeights(self): return self._export("PFPC_WEIGHT")
    def exportMFNCWeights(self): return self._export("MFNC_WEIGHT")


class CBMSimCore:
    """CBMSimCore (CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/interface/cbmsimcore.h:32-75).

    ``mzoneRSeed`` keys each microzone's NC->IO release draws; ``device`` is
    the GPU that holds the whole network; ``resident_steps`` reserves HBM for
    that many steps of MF input used by :meth:`run`.
    """

    def __init__(self, state, mzoneRSeed=None, device=0, resident_steps=0):
        self.state = state
        self._h = ctypes.c_void_p()
        seeds = None if mzoneRSeed is None else np.asarray(mzoneRSeed, dtype=np.int32)
        if resident_steps:
            _check(lib.cbm_sim_create_resident(state._h, _ptr(seeds), device, resident_steps, ctypes.byref(self._h)))
        else:
            _check(lib.cbm_sim_create(state._h, _ptr(seeds), device, ctypes.byref(self._h)))
        self._innet = InNet(self, 0)
        self._zones = [MZone(self, z) for z in range(state.getNumZones())]

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.cbm_sim_destroy(self._h)
            self._h = ctypes.c_void_p()

    def close(self):
        self.__del__()

    def calcActivity(self):
        _check(lib.cbm_sim_calc_activity(self._h))

    def updateMFInput(self, mf):
        mf = np.ascontiguousarray(mf, dtype=np.uint8)
        _check(lib.cbm_sim_update_mf(self._h, mf.ctypes.data))

    def updateErrDrive(self, zoneN, errDriveRelative):
        _check(lib.cbm_sim_update_err_drive(self._h, zoneN, errDriveRelative))

    def writeToState(self, path=None):
        """writeToState(): the device state back into the CBMState;
        writeToState(fstream&): then saved to a file name, or into a binary
        file object at its position."""
        if path is None:
            _check(lib.cbm_sim_write_to_state(self._h))
        elif hasattr(path, "write"):
            path.write(_serialised(lambda d, c, n: lib.cbm_sim_save_mem(self._h, d, c, n)))
        else:
            _check(lib.cbm_sim_save(self._h, os.fsencode(path)))

    def getInputNet(self):
        return self._innet

    def getMZoneList(self):
        return self._zones

    # ---- beyond the reference API: resident input, graph-captured runs
    def steps_done(self):
        v = ctypes.c_uint64()
        _check(lib.cbm_sim_steps_done(self._h, ctypes.byref(v)))
        return v.value

    def mf_words(self):
        v = ctypes.c_uint32()
        _check(lib.cbm_sim_mf_words(self._h, ctypes.byref(v)))
        return v.value

    def load_mf_stream(self, bits):
        bits = np.ascontiguousarray(bits, dtype=np.uint32)
        _check(lib.cbm_sim_load_mf_stream(self._h, _ptr(bits), bits.shape[0]))

    def run(self, nsteps, chunk=50, time_pass=False):
        ms, pms = ctypes.c_float(), ctypes.c_float()
        _check(lib.cbm_sim_run(self._h, nsteps, chunk, ctypes.byref(ms), ctypes.byref(pms) if time_pass else None))
        return ms.value, (pms.value if time_pass else None)

    def last_tail_ms(self):
        ms = ctypes.c_float()
        _check(lib.cbm_sim_last_tail_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def timer_start(self):
        _check(lib.cbm_sim_timer_start(self._h))

    def timer_stop(self):
        ms = ctypes.c_float()
        _check(lib.cbm_sim_timer_stop(self._h, ctypes.byref(ms)))
        return ms.value

    def algorithmic_bytes_per_step(self):
        return lib.cbm_sim_algorithmic_bytes_per_step(self._h)

    def set_eyelid_protocol(self, rates, **protocol):
        """Drive the next steps with the device eyelid protocol
        (cbm_sim_set_eyelid_protocol); rates is [3, numMF] Hz (background, CS
        tonic, CS phasic); keyword fields as cbm_eyelid_protocol."""
        rates = np.ascontiguousarray(rates, dtype=np.float32)
        p = EyelidProtocol.from_fields(rates, protocol)
        _check(lib.cbm_sim_set_eyelid_protocol(self._h, ctypes.byref(p)))
        self._protocol = protocol

    def set_statevar_input(self, coding, values, mfSeed=0, mfThreshDecayTau=4.0):
        """Drive the MF input from the next step on by the state-variable
        coding on the device (cbm_sim_set_statevar_input): coding is a
        networks.StateVariableMF (its fibre assignment, preferred values,
        width and rates), values the environment's state, [steps, numVars],
        used row by row and cyclically."""
        values = np.ascontiguousarray(values, dtype=np.float32)
        if values.ndim != 2 or values.shape[1] != coding.n_vars:
            raise ValueError("values must be [steps, numVars]")
        mean = np.ascontiguousarray(coding.mean, dtype=np.float32)
        relaxed = np.ascontiguousarray(coding.relaxed, dtype=np.float32)
        excited = np.ascontiguousarray(coding.excited, dtype=np.float32)
        c = StateVarInput(numVars=coding.n_vars, fibresPerVar=coding.per, lo=float(coding.lo), hi=float(coding.hi),
                          den=float(coding._den), norm=float(coding._norm), maxPossible=float(coding._max_possible),
                          mean=mean.ctypes.data, relaxed=relaxed.ctypes.data, excited=excited.ctypes.data,
                          values=values.ctypes.data, numSteps=values.shape[0], mfSeed=mfSeed,
                          mfThreshDecayTau=mfThreshDecayTau)
        _check(lib.cbm_sim_set_statevar_input(self._h, ctypes.byref(c)))
        self._protocol = None

    def statevar_rates(self, row):
        """The MF rates (Hz) the device computes for row `row` of the
        running state-variable input's values."""
        out = np.empty(self.state.con("numMF"), dtype=np.float32)
        _check(lib.cbm_sim_statevar_rates(self._h, row, out.ctypes.data))
        return out

    def record_gr(self):
        """Record the running protocol's GR peri-stimulus histogram on the
        device from the next step on (cbm_sim_record_gr)."""
        _check(lib.cbm_sim_record_gr(self._h))

    def record_trial_data(self):
        """Record the running protocol's ECTrialsData histograms and rasters
        on the device from the next step on (cbm_sim_record_trial_data)."""
        _check(lib.cbm_sim_record_trial_data(self._h))

    def trial_data(self):
        """The ECTrialsData records (after record_trial_data):
        {"psh": {name: f32 [bins, cells]}, "raster": {name: u32 [trials,
        window steps // 32, cells]}, "eyelid": f32 [trials, window steps]}
        under the eyelid driver's names; "eyelid" is the driver's smoothed
        trace (eyelid_out of the raw integrator output)."""
        if not lib.cbm_sim_trial_record_bytes(self._h, TRIAL_PSH["go"][0]):
            raise CBMError(1, "the trial data is not recorded")
        p = self._protocol
        rows = (p["csOff"] + p["postCS"] - (p["csOn"] - p["preCS"])) // 32
        out = {"psh": {}, "raster": {}, "eyelid": eyelid_out(self.trial_record("eyelid"))}
        for kinds, key, dtype in ((TRIAL_PSH, "psh", np.float32), (TRIAL_RASTER, "raster", np.uint32)):
            for name, (k, cell) in kinds.items():
                cells = self.state.con(cell)
                n = lib.cbm_sim_trial_record_bytes(self._h, k)
                a = np.empty(n // 4, dtype=dtype)
                if n:  # rasters of a protocol that keeps no trial are empty
                    _check(lib.cbm_sim_trial_record(self._h, k, a.ctypes.data, n))
                out[key][name] = a.reshape(-1, cells) if key == "psh" else a.reshape(p["numDataTrials"], rows, cells)
        return out

    def write_trial_data(self, path):
        """The eyelid driver's data file (ECTrialsData::writeData) of the
        running protocol's records, after record_gr and record_trial_data and
        a run over all kept trials (trialdata.write_ec_trials_data)."""
        from .trialdata import write_ec_trials_data
        write_ec_trials_data(path, self.trial_data(), self.trial_record("gr"), self.trial_record("eyelid"),
                             self._protocol, self.state.con("numGR"), int(self.state.act("msPerTimeStep")))

    def write_session(self, path, mf_population=None):
        """ECManagementDelay::writeDataToFile (Eyelid_Sim_CBM_Dev/src/ectrial/
        ecmanagementdelay.cpp:275-290): the state, then the driver's data
        file, in one file (the driver reads it back with CBMState(fstream&)
        and ECTrialsData(fstream&)); with mf_population (networks.MFPopulation)
        also its tables in path + "_MFPop"."""
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            td = os.path.join(d, "data")
            self.write_trial_data(td)
            with open(path, "wb") as out:
                self.writeToState(out)
                with open(td, "rb") as f:
                    out.write(f.read())
        if mf_population is not None:
            mf_population.write(path + "_MFPop")

    def trial_record(self, kind):
        """Records of the running protocol: 'nc' / 'pc' spike counts
        [trials, bins, cells] (u32), 'eyelid' [trials, window steps] (f32), or
        'gr' [bins, numGR] (u16, the kept trials summed; after record_gr)."""
        k = {"nc": 0, "pc": 1, "eyelid": 2, "gr": 3}[kind]
        n = lib.cbm_sim_trial_record_bytes(self._h, k)
        if not n:
            raise CBMError(1, "no protocol is running" if kind != "gr" else "the GR histogram is not recorded")
        if kind == "gr":
            out = np.empty(n // 2, dtype=np.uint16)
            _check(lib.cbm_sim_trial_record(self._h, k, out.ctypes.data, n))
            return out.reshape(-1, self.state.con("numGR"))
        out = np.empty(n // 4, dtype=np.float32 if kind == "eyelid" else np.uint32)
        _check(lib.cbm_sim_trial_record(self._h, k, out.ctypes.data, n))
        p = self._protocol
        trials = max(1, p["numDataTrials"])
        if kind == "eyelid":
            return out.reshape(trials, -1)
        return out.reshape(trials, -1, self.state.con("numNC" if kind == "nc" else "numPC"))

    def run_flushed(self, nsteps, flush_bytes):
        """nsteps steps, each after an L2 flush (a write of flush_bytes); the
        summed device time of the steps alone, in ms."""
        ms = ctypes.c_float()
        _check(lib.cbm_sim_run_flushed(self._h, nsteps, flush_bytes, ctypes.byref(ms)))
        return ms.value

    def run_flushed_kernels(self, nsteps, flush_bytes):
        """nsteps steps after an L2 flush each, the two step kernels timed
        separately: (mean GR-pass ms, mean small-cell kernel ms)."""
        p, t = ctypes.c_float(), ctypes.c_float()
        _check(lib.cbm_sim_run_flushed_kernels(self._h, nsteps, flush_bytes, ctypes.byref(p), ctypes.byref(t)))
        return p.value, t.value

    def layout_bytes_per_step(self):
        return lib.cbm_sim_layout_bytes_per_step(self._h)

    def pass_geometry(self):
        """(kernel name, consumer warps, rows per stage, stages) of the GR pass."""
        v = [ctypes.c_uint32() for _ in range(4)]
        _check(lib.cbm_sim_pass_geometry(self._h, *[ctypes.byref(x) for x in v]))
        return _pass_kind_name(v[0].value, single=True), v[1].value, v[2].value, v[3].value


def _pass_kind_name(kind, single):
    """Kernel name of a GR-pass kind (cbm_sim_pass_geometry's *kind)."""
    if kind == 3 and not single:
        return "grPassVecBatchKernel"
    return ("grPassKernel", "grPassTmaKernel", "grPassPersistentKernel", "grPassVecKernel")[kind]


class CBMBatch:
    """Independent networks advanced together (cbm_batch_*): one GR-pass
    launch over all of them per step, each driven by its own device protocol."""

    def __init__(self, states, mzoneRSeeds=None, device=0):
        self.states = list(states)
        arr = (ctypes.c_void_p * len(self.states))(*[st._h for st in self.states])
        seeds = None
        if mzoneRSeeds is not None:
            seeds = np.ascontiguousarray(np.concatenate([np.atleast_1d(np.asarray(x, dtype=np.int32))
                                                          for x in mzoneRSeeds]), dtype=np.int32)
        self._h = ctypes.c_void_p()
        self._protocols = [None] * len(self.states)
        _check(lib.cbm_batch_create(arr, len(self.states), _ptr(seeds), device, ctypes.byref(self._h)))

    def __del__(self):
        if getattr(self, "_h", None):
            lib.cbm_batch_destroy(self._h)
            self._h = None

    def close(self):
        self.__del__()

    def set_eyelid_protocol(self, i, rates, **protocol):
        rates = np.ascontiguousarray(rates, dtype=np.float32)
        p = EyelidProtocol.from_fields(rates, protocol)
        _check(lib.cbm_batch_set_eyelid_protocol(self._h, i, ctypes.byref(p)))
        self._protocols[i] = protocol

    def run(self, nsteps, chunk=50):
        ms = ctypes.c_float()
        _check(lib.cbm_batch_run(self._h, nsteps, chunk, ctypes.byref(ms)))
        return ms.value

    def pass_geometry(self):
        """(kernel name, consumer warps, rows per stage, stages) of the batch's GR pass."""
        v = [ctypes.c_uint32() for _ in range(4)]
        _check(lib.cbm_batch_pass_geometry(self._h, *[ctypes.byref(x) for x in v]))
        return _pass_kind_name(v[0].value, single=len(self.states) == 1), v[1].value, v[2].value, v[3].value

    def autotune(self, nsteps=100):
        """Time every GR-pass geometry on a scratch copy; keep the fastest.
        Returns (\"kind,W,RW,S,B,M\", ms)."""
        buf = ctypes.create_string_buffer(64)
        ms = ctypes.c_float()
        _check(lib.cbm_batch_autotune(self._h, nsteps, buf, 64, ctypes.byref(ms)))
        return buf.value.decode(), ms.value

    def trial_record(self, i, kind):
        k = {"nc": 0, "pc": 1, "eyelid": 2}[kind]
        n = lib.cbm_batch_trial_record_bytes(self._h, i, k)
        if not n:
            raise CBMError(1, "no protocol is running on that instance")
        out = np.empty(n // 4, dtype=np.float32 if kind == "eyelid" else np.uint32)
        _check(lib.cbm_batch_trial_record(self._h, i, k, out.ctypes.data, n))
        trials = max(1, self._protocols[i]["numDataTrials"])
        if kind == "eyelid":
            return out.reshape(trials, -1)
        return out.reshape(trials, -1, self.states[i].con("numNC" if kind == "nc" else "numPC"))

    def record_trial_data(self, i):
        """Record instance i's ECTrialsData from the next step on
        (cbm_batch_record_trial_data)."""
        _check(lib.cbm_batch_record_trial_data(self._h, i))

    def trial_data(self, i):
        """Instance i's ECTrialsData records, in the form of
        CBMSimCore.trial_data (after record_trial_data)."""
        p = self._protocols[i]
        if not lib.cbm_batch_trial_record_bytes(self._h, i, TRIAL_PSH["go"][0]):
            raise CBMError(1, "the trial data of that instance is not recorded")
        rows = (p["csOff"] + p["postCS"] - (p["csOn"] - p["preCS"])) // 32
        out = {"psh": {}, "raster": {}, "eyelid": eyelid_out(self.trial_record(i, "eyelid"))}
        for kinds, key, dtype in ((TRIAL_PSH, "psh", np.float32), (TRIAL_RASTER, "raster", np.uint32)):
            for name, (k, cell) in kinds.items():
                cells = self.states[i].con(cell)
                n = lib.cbm_batch_trial_record_bytes(self._h, i, k)
                a = np.empty(n // 4, dtype=dtype)
                if n:
                    _check(lib.cbm_batch_trial_record(self._h, i, k, a.ctypes.data, n))
                out[key][name] = a.reshape(-1, cells) if key == "psh" else a.reshape(p["numDataTrials"], rows, cells)
        return out

    def writeToState(self, i, path=None):
        _check(lib.cbm_batch_write_to_state(self._h, i))
        if path is not None:
            self.states[i].writeState(path)

    def num_gr(self):
        return lib.cbm_batch_num_gr(self._h)


_PROTOCOL_FIELDS = [("trialSteps", ctypes.c_uint32), ("csOn", ctypes.c_int32), ("csOff", ctypes.c_int32),
                    ("csPhasicOff", ctypes.c_int32), ("csStartTrial", ctypes.c_uint32),
                    ("plastOnDelay", ctypes.c_int32), ("plastOffDelay", ctypes.c_int32),
                    ("plastLTD", ctypes.c_float), ("plastLTP", ctypes.c_float), ("usErrDrive", ctypes.c_float),
                    ("mfSeed", ctypes.c_int32), ("mfThreshDecayTau", ctypes.c_float),
                    ("mfFreqBG", ctypes.c_void_p), ("mfFreqCSTonic", ctypes.c_void_p),
                    ("mfFreqCSPhasic", ctypes.c_void_p), ("dataStartTrial", ctypes.c_uint32),
                    ("numDataTrials", ctypes.c_uint32), ("preCS", ctypes.c_int32), ("postCS", ctypes.c_int32),
                    ("binSteps", ctypes.c_uint32), ("eyeGDecayTau", ctypes.c_float), ("eyeGInc", ctypes.c_float),
                    ("eyeGShift", ctypes.c_float), ("eyeGLeakRaw", ctypes.c_float), ("eyeMaxAmp", ctypes.c_float)]


class StateVarInput(ctypes.Structure):
    """cbm_statevar_input (include/cbm_b200.h)."""
    _fields_ = [("numVars", ctypes.c_uint32), ("fibresPerVar", ctypes.c_uint32), ("lo", ctypes.c_float),
                ("hi", ctypes.c_float), ("den", ctypes.c_float), ("norm", ctypes.c_double),
                ("maxPossible", ctypes.c_float), ("mean", ctypes.c_void_p), ("relaxed", ctypes.c_void_p),
                ("excited", ctypes.c_void_p), ("values", ctypes.c_void_p), ("numSteps", ctypes.c_uint64),
                ("mfSeed", ctypes.c_int32), ("mfThreshDecayTau", ctypes.c_float)]


class EyelidProtocol(ctypes.Structure):
    """cbm_eyelid_protocol (include/cbm_b200.h)."""
    _fields_ = _PROTOCOL_FIELDS

    @classmethod
    def from_fields(cls, rates, fields):
        p = cls(**{n: fields[n] for n, _ in _PROTOCOL_FIELDS if not n.startswith("mfFreq")})
        p.mfFreqBG = rates[0].ctypes.data
        p.mfFreqCSTonic = rates[1].ctypes.data
        p.mfFreqCSPhasic = rates[2].ctypes.data
        p._rates = rates  # keeps the tables alive during the call
        return p


def eyelid_protocol_defaults(state, **kw):
    """The reference eyelid driver's settings (ecmanagementdelay.cpp:90-170,
    201-235) for 5000-step trials with the CS at 2000-2500 ms: LTD step
    -0.0005 x the LTD/LTP ratio ((csOff - csOn + msLTDStartAPIO) /
    msLTDDurationIO, at least 0.5), LTP step 0.0005, eyelid integrator
    (10.5, 0.012, -0.13, 0.13, 100), recording window 500 ms either side."""
    p = dict(trialSteps=5000, csOn=2000, csOff=2500, csPhasicOff=2000, csStartTrial=0, plastOnDelay=200,
             plastOffDelay=200, usErrDrive=1.0, mfSeed=0, mfThreshDecayTau=4.0, dataStartTrial=0,
             numDataTrials=1, preCS=500, postCS=500, binSteps=10, eyeGDecayTau=10.5, eyeGInc=0.012,
             eyeGShift=-0.13, eyeGLeakRaw=0.13, eyeMaxAmp=100.0, plastLTP=0.0005)
    p.update(kw)
    if "plastLTD" not in p:
        ratio = ((p["csOff"] - p["csOn"]) + state.act("msLTDStartAPIO")) / state.act("msLTDDurationIO")
        p["plastLTD"] = -0.0005 * max(ratio, 0.5)
    return p


def mf_bits(mf_bytes, words):
    """Pack [steps, numMF] spike bytes into [steps, words] uint32 bit rows."""
    mf = np.asarray(mf_bytes, dtype=np.uint8) != 0
    steps, n = mf.shape
    pad = np.zeros((steps, words * 32), dtype=bool)
    pad[:, :n] = mf
    return np.ascontiguousarray(np.packbits(pad, axis=1, bitorder="little").view("<u4")).astype(np.uint32)


def device_expf(x, device=0):
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    _check(lib.cbm_device_expf(device, _ptr(x), _ptr(out), x.size))
    return out


def device_exp(x, device=0):
    """The device's double exp (cbm_device_exp) of float64 values."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    _check(lib.cbm_device_exp(device, _ptr(x), _ptr(out), x.size))
    return out
