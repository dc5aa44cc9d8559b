"""The eyelid driver's data file from device records.

``write_ec_trials_data`` lays out a run's trial records the way the
reference's ECTrialsData::writeData writes its own
(CBM_DATA_LIB_DEV/src/interfaces/ectrialsdata.cpp): a text header line, the
eyelid record (EyelidOut::writeData, outdata/eyelidout.cpp), every
peri-stimulus histogram (PeriStimHistFloat::writeData,
peristimhist/peristimhistfloat.cpp) and every raster
(ISpikeRaster / SpikeRasterBitArray::writeData, spikeraster/
spikerasterbitarray.cpp) in the order of the reference's std::map (byte
order of the names), then the count of raw-uint records (none).  The
histogram and raster sets are those the eyelid driver builds
(Eyelid_Sim_CBM_Dev/src/ectrial/ecmanagementdelay.cpp:107-156); its "gr"
histogram covers the first numGR / 10 cells.

The counters written with each record are those of a run whose kept trials
were all recorded to their end, which is what the driver writes at the end
of a session.
"""
import numpy as np


def _line(*values):
    return (" ".join(str(int(v)) for v in values) + "\n").encode()


def write_ec_trials_data(path, trial_data, gr_psh, eyelid_raw, proto, num_gr, ms_per_step=1, num_ts_smooth=4):
    """Write the driver's data file.

    trial_data: {"psh": {name: f32 [bins, cells]}, "raster": {name: u32
    [trials, rows, cells]}} (CBMSimCore.trial_data); gr_psh: [bins, numGR]
    GR counts (CBMSimCore.trial_record("gr")); eyelid_raw: the integrator's
    output [trials, window steps] (trial_record("eyelid")); proto: the
    protocol's fields (preCS, postCS, csOn, csOff, binSteps,
    numDataTrials)."""
    from . import eyelid_out
    pre, post = int(proto["preCS"]), int(proto["postCS"])
    cs = int(proto["csOff"]) - int(proto["csOn"])
    nd, bin_steps = int(proto["numDataTrials"]), int(proto["binSteps"])
    ms_total = pre + cs + post
    ts_total = ms_total // ms_per_step
    n_bins = -(-ts_total // bin_steps)
    psh = dict(trial_data["psh"])
    psh["gr"] = np.asarray(gr_psh)[:, : num_gr // 10].astype(np.float32)
    rows = ts_total // 32
    with open(path, "wb") as f:
        f.write(_line(pre, cs, post, ms_total, ms_per_step, ts_total, nd))
        # EyelidOut: every kept trial recorded to its end
        f.write(_line(nd, ms_per_step, num_ts_smooth, ms_total, ts_total, nd, 0))
        f.write(np.ascontiguousarray(eyelid_out(eyelid_raw, num_ts_smooth), dtype=np.float32).tobytes())
        f.write(_line(len(psh)))
        for name in sorted(psh):
            h = np.ascontiguousarray(psh[name], dtype=np.float32)
            if h.shape[0] != n_bins:
                raise ValueError(f"histogram {name}: {h.shape[0]} bins, the window has {n_bins}")
            f.write(name.encode() + b"\n")
            f.write(_line(h.shape[1], ts_total, bin_steps, n_bins, 0, nd))
            f.write(h.tobytes())
        rasters = trial_data["raster"]
        updates = nd * ((ts_total - 1) // 32)
        cur_trial, cur_buf = (updates // rows, updates % rows) if rows else (0, 0)
        f.write(_line(len(rasters)))
        for name in sorted(rasters):
            r = np.ascontiguousarray(rasters[name], dtype=np.uint32)
            f.write(name.encode() + b"\n")
            f.write(name.encode() + b" " + _line(r.shape[2], nd, ms_total).rstrip(b"\n") + b" ")
            f.write(_line(ms_per_step, cur_trial, 32 * cur_buf, cur_buf, ts_total, rows))
            f.write(r.tobytes())
        f.write(_line(0))


class _Reader:
    """Whitespace-separated numbers and names, then raw bytes after one
    separator character, as the reference's fstream readers take them
    (operator>> then seekg(1, ios::cur))."""

    def __init__(self, buf, pos=0):
        self.buf, self.pos = buf, pos

    def word(self):
        b = self.buf
        while b[self.pos: self.pos + 1].isspace():
            self.pos += 1
        start = self.pos
        while self.pos < len(b) and not b[self.pos: self.pos + 1].isspace():
            self.pos += 1
        if start == self.pos:
            raise ValueError("trial data file truncated")
        return b[start: self.pos].decode()

    def ints(self, n):
        return [int(self.word()) for _ in range(n)]

    def raw(self, dtype, count):
        self.pos += 1  # the separator after the header line
        nbytes = np.dtype(dtype).itemsize * count
        if self.pos + nbytes > len(self.buf):
            raise ValueError("trial data file truncated")
        a = np.frombuffer(self.buf, dtype=dtype, count=count, offset=self.pos).copy()
        self.pos += nbytes
        return a


def read_ec_trials_data(buf, pos=0):
    """Parse a data file of ECTrialsData::writeData starting at byte pos
    (ECTrialsData(fstream &), ectrialsdata.cpp): {"header": {...},
    "eyelid": f32 [trials, steps], "psh": {name: f32 [bins, cells]},
    "psh_trials": {name: trials recorded}, "psh_bin_steps": {name: steps a
    bin}, "raster": {name: u32 [trials, rows, cells]}, "raster_trials":
    {name: the raster's completed trials, its curTrialN}}."""
    r = _Reader(buf, pos)
    pre, cs, post, ms_total, ms_per_ts, ts_total, n_trials = r.ints(7)
    out = {"header": dict(msPreCS=pre, msCS=cs, msPostCS=post, msTotal=ms_total, msPerTimeStep=ms_per_ts,
                          tsTotal=ts_total, numTrials=n_trials), "psh": {}, "psh_trials": {},
           "psh_bin_steps": {}, "raster": {}, "raster_trials": {}}
    e_trials, _, _, _, e_ts, _, _ = r.ints(7)
    out["eyelid"] = r.raw(np.float32, e_trials * e_ts).reshape(e_trials, e_ts)
    for _ in range(r.ints(1)[0]):
        name = r.word()
        cells, _, bin_steps, bins, _, trials = r.ints(6)
        out["psh"][name] = r.raw(np.float32, bins * cells).reshape(bins, cells)
        out["psh_trials"][name] = trials
        out["psh_bin_steps"][name] = bin_steps
    for _ in range(r.ints(1)[0]):
        name = r.word()
        r.word()  # the raster's own copy of its name
        cells, trials, _ = r.ints(3)
        _, cur_trial, _, _, _, rows = r.ints(6)
        out["raster"][name] = r.raw(np.uint32, trials * rows * cells).reshape(trials, rows, cells)
        out["raster_trials"][name] = cur_trial
    if r.ints(1)[0] != 0:
        raise ValueError("raw-uint records are not read")
    out["end"] = r.pos + (buf[r.pos: r.pos + 1] == b"\n")  # past the count's line end
    return out


def read_session(path):
    """The driver's session file (writeDataToFile): (CBMState, trial data)
    as ECManagementDelay's resume constructor reads it
    (ecmanagementdelay.cpp:26-50)."""
    from . import CBMState
    with open(path, "rb") as f:
        state = CBMState(f)  # leaves f just after the state, like CBMState(fstream&)
        state_bytes = f.tell()
        f.seek(0)
        buf = f.read()
    return state, read_ec_trials_data(buf, state_bytes)


class PeriStimHist:
    """PeriStimHistFloat's getters (peristimhist/peristimhistfloat.cpp) over
    one histogram [bins, cells]."""

    def __init__(self, counts, steps_per_bin, trials):
        self.counts = np.asarray(counts, dtype=np.float32)
        self.steps_per_bin, self.trials = int(steps_per_bin), int(trials)

    def getCellPSH(self, cellN):
        return [float(v) for v in self.counts[:, cellN]]

    def getPopPSHs(self):
        return [self.getCellPSH(i) for i in range(self.getNumCells())]

    def getNumCells(self):
        return self.counts.shape[1]

    def getNumBins(self):
        return self.counts.shape[0]

    def getBinWidthInMS(self):
        return self.steps_per_bin

    def getNumTrials(self):
        return self.trials


class SpikeRaster:
    """SpikeRasterBitArray's getters (spikeraster/spikerasterbitarray.cpp:
    82-170) over one raster [trials, rows, cells] of 32-step apBuf words:
    bit 31 of a row is its earliest step."""

    def __init__(self, words, ms_per_step=1, trials_done=None):
        self.words = np.asarray(words, dtype=np.uint32)
        self.ms_per_step = int(ms_per_step)
        self.trials_done = self.words.shape[0] if trials_done is None else int(trials_done)

    def getNumCells(self):
        return self.words.shape[2]

    def getNumTrials(self):
        return self.trials_done

    def getUpdateInterval(self):
        return 32

    def getCellSpikeTimes(self, cellN, trialN=None, offset=0):
        """Spike times of a cell in one trial, or (trialN None, the
        reference's two-argument form) in every recorded trial."""
        if trialN is None:
            return [self.getCellSpikeTimes(cellN, t, offset) for t in range(self.trials_done)]
        times, t = [], offset
        for w in self.words[trialN, :, cellN]:
            for j in range(32):
                if (int(w) << j) & 0x80000000:
                    times.append(t)
                t += self.ms_per_step
        return times

    def getPopSpikesAtTS(self, timeStep, trialN):
        row, bit = divmod(int(timeStep), 32)
        if row >= self.words.shape[1]:
            return [False] * self.getNumCells()
        return [bool(w & (0x80000000 >> bit)) for w in self.words[trialN, row]]


class TrialsData:
    """ECTrialsData's getters (interfaces/ectrialsdata.cpp) over a data
    file (``from_file``) or a simulator's records (``from_sim``)."""

    def __init__(self, parsed):
        self._d = parsed
        h = parsed["header"]
        self._ms_per_step = h["msPerTimeStep"]

    @classmethod
    def from_file(cls, path, offset=0):
        with open(path, "rb") as f:
            return cls(read_ec_trials_data(f.read(), offset))

    @classmethod
    def from_sim(cls, sim):
        import os
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "data")
            sim.write_trial_data(p)
            return cls.from_file(p)

    def getPSH(self, cellT):
        return PeriStimHist(self._d["psh"][cellT], self._d["psh_bin_steps"][cellT], self._d["psh_trials"][cellT])

    def getRaster(self, cellT):
        # getNumTrials and the all-trials spike times count the raster's
        # completed trials (SpikeRasterBitArray's curTrialN), which fall
        # behind the allocated trials when the window is a multiple of 32 steps
        return SpikeRaster(self._d["raster"][cellT], self._ms_per_step,
                           trials_done=self._d.get("raster_trials", {}).get(cellT))

    def getEyelidData(self, trialN):
        return [float(v) for v in self._d["eyelid"][trialN]]

    def getTSPerRasterUpdate(self):
        return 32 if self._d["raster"] else 0

    def getMSPreTrial(self):
        return self._d["header"]["msPreCS"]

    def getMSTrial(self):
        return self._d["header"]["msCS"]

    def getMSPostTrial(self):
        return self._d["header"]["msPostCS"]

    def getMSPerTimeStep(self):
        return self._ms_per_step

    def getMSTotal(self):
        return self._d["header"]["msTotal"]

    def getTimeStepsTotal(self):
        return self._d["header"]["tsTotal"]

    def getMaxNumTrials(self):
        return self._d["header"]["numTrials"]
