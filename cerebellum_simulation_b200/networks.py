"""Network construction and mossy-fibre (MF) input for the benchmark configurations.

The reference builds networks with a spatial glomerulus-mediated generator
(CBM_STATE_LIB_DEV/src/state/innetconnectivitystate.cpp:716-962).  The
configurations this package is measured on are defined with random wiring
instead ("each GR with 4 random MF and 3 random GO dendrites", "each GO
receiving N random GR"), so they are built here: the input-net tables are
filled in the reference's own layouts (cell-major, counts plus index lists),
the axonal delay masks follow assignGRDelays (innetconnectivitystate.cpp:
920-962), GO->GO wiring follows connectGOGO's local-matrix rule (:852-918)
and the microzone wiring and initial activity come from cbm_state_new.  The
result is an ordinary CBMState: it can be saved in the reference's format and
loaded by the reference.

MF spikes follow the reference's regenerating Poisson rule
(CBM_TOOLS_LIB_DEV/src/poissonregencells.cpp:49-66) driven by the package's
counter-based stream (cbm_rng.hpp), so any MF sequence can be regenerated
from (seed, step, fibre).
"""
import ctypes
import ctypes.util
import math
import os

import numpy as np

PARAMS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "params")

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
STREAM_MF = 0x4D46494E
STREAM_WIRING = 0x57495245


def act_params(name):
    """Text of a bundled activity-parameter set ("16k" or "dense")."""
    with open(os.path.join(PARAMS_DIR, f"act_{name}.txt")) as f:
        return f.read()


def _libm_expf(x):
    """The C library's expf (numpy's float32 exp rounds differently)."""
    global _EXPF
    if _EXPF is None:
        libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
        libm.expf.restype = ctypes.c_float
        libm.expf.argtypes = [ctypes.c_float]
        _EXPF = libm.expf
    return np.float32(_EXPF(x))


_EXPF = None


def splitmix64(x):
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def uniform24(seed, stream, counter):
    """Same values as cbm::rng::uniform24 (float32 in [0,1), 24 random bits)."""
    key = splitmix64(np.uint64((int(seed) & 0xFFFFFFFF) << 32 | (stream & 0xFFFFFFFF)))
    h = splitmix64(key ^ np.asarray(counter, dtype=np.uint64))
    return (h >> np.uint64(40)).astype(np.float32) * np.float32(1.0 / 16777216.0)


class RegenPoissonMF:
    """PoissonRegenCells (poissonregencells.cpp:10-66) over numMF fibres.

    threshDecay = 1 - exp(-msPerTS/threshDecayTau) (in float: the reference's
    exp of a float argument is C++'s float overload, the C library's expf) and
    the per-step rule thresh += (1-thresh)*threshDecay; ap = U < (freq*sPerTS)
    *thresh; thresh = (!ap)*thresh, in float32.
    """

    def __init__(self, num_mf, seed, thresh_decay_tau=4.0, ms_per_step=1.0):
        self.n = num_mf
        self.seed = seed
        ms = np.float32(ms_per_step)
        self.s_per_ts = np.float32(ms / np.float32(1000))
        # threshDecay = 1 - exp(-msPerTS / tau): a float quotient, the C library's expf, a float subtraction
        self.thresh_decay = np.float32(np.float32(1) - _libm_expf(float(np.float32(-ms / np.float32(thresh_decay_tau)))))
        self.thresh = np.ones(num_mf, dtype=np.float32)
        self.t = 0

    def step(self, freqs):
        freqs = np.asarray(freqs, dtype=np.float32)
        self.t += 1
        one = np.float32(1)
        self.thresh = (self.thresh + (one - self.thresh) * self.thresh_decay).astype(np.float32)
        ctr = (np.uint64(self.t) << np.uint64(20)) | np.arange(self.n, dtype=np.uint64)
        u = uniform24(self.seed, STREAM_MF, ctr)
        ap = u < ((freqs * self.s_per_ts).astype(np.float32) * self.thresh).astype(np.float32)
        self.thresh = np.where(ap, np.float32(0), self.thresh).astype(np.float32)
        return ap.astype(np.uint8)

    def run(self, freqs_fn, steps):
        out = np.empty((steps, self.n), dtype=np.uint8)
        for s in range(steps):
            out[s] = self.step(freqs_fn(self.t + 1))
        return out


def _distinct_choice(rng, n_rows, k, high):
    """n_rows rows of k distinct integers in [0, high)."""
    out = rng.integers(0, high, size=(n_rows, k), dtype=np.int64)
    for _ in range(64):
        s = np.sort(out, axis=1)
        dup = np.any(s[:, 1:] == s[:, :-1], axis=1) if k > 1 else np.zeros(n_rows, bool)
        if not dup.any():
            return out
        out[dup] = rng.integers(0, high, size=(int(dup.sum()), k), dtype=np.int64)
    raise RuntimeError("could not draw distinct indices")


def _gr_lists_from_targets(targets_of_src, n_gr, max_slots=None):
    """Invert per-source GR target rows into per-GR source lists (ascending source)."""
    src = np.repeat(np.arange(targets_of_src.shape[0], dtype=np.int64), targets_of_src.shape[1])
    gr = targets_of_src.ravel()
    order = np.lexsort((src, gr))
    gr, src = gr[order], src[order]
    counts = np.bincount(gr, minlength=n_gr)
    slots = int(counts.max()) if max_slots is None else max_slots
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    pos = np.arange(gr.size) - starts[gr]
    table = np.full((n_gr, max(slots, 1)), 0xFFFFFFFF, dtype=np.uint32)
    table[gr, pos] = src
    return table, counts.astype(np.int32), slots


def con_params_text(gr_xp2, gr_yp2, go_xp2, go_yp2, mf_p2, *, max_gr_out, max_mf_go_per_mf,
                    vel, af_delay=1, sc_p2=9, pc_p2=5, nc_p2=3, io_p2=2, pcnc=3,
                    gogo=((0, -1, 1.0), (-1, -1, 1.0), (-1, 0, 1.0), (-1, 1, 1.0)), coup=None):
    """Connectivity-parameter text in the reference's key/value format
    (ConnectivityParams(fstream&), connectivityparams.cpp:12-88).  The
    glomerulus layer is sized so that the MF->GO out-list holds
    max_mf_go_per_mf entries per fibre (numpMFfromMFtoGL * maxnumpGLfromGLtoGO)."""
    gl_p2 = mf_p2 + max(0, int(np.ceil(np.log2(max(1, max_mf_go_per_mf)))))
    lines = [
        f"glXP2 {gl_p2 - gl_p2 // 2}", f"glYP2 {gl_p2 // 2}",
        "maxnumpGLfromGLtoGR 1", "lownumpGLfromGLtoGR 1", "maxnumpGLfromGLtoGO 1", "maxnumpGLfromGOtoGL 1",
        f"numMFP2 {mf_p2}", f"goXP2 {go_xp2}", f"goYP2 {go_yp2}",
        "maxnumpGOfromGRtoGO 1", "maxnumpGOfromGLtoGO 1", "maxnumpGOfromGOtoGL 1",
        "spanGODecDenOnGLX 1", "spanGODecDenOnGLY 1", "spanGOAscDenOnGRX 1", "spanGOAscDenOnGRY 1",
        "spanGOAxonOnGLX 1", "spanGOAxonOnGLY 1",
        "GOGOLocalMatrix", f"maxnumpGOInfromGOtoGO {len(gogo)}", f"maxnumpGOOutfromGOtoGO {len(gogo)}",
    ]
    lines += [f"{a} {b} {c}" for a, b, c in gogo]
    if coup:
        lines += ["GOGOCoupLocalMatrix", f"maxnumpGOCoupInfromGOtoGO {len(coup)}",
                  f"maxnumpGOCoupOutfromGOtoGO {len(coup)}"]
        lines += [f"{a} {b} {c}" for a, b, c in coup]
    lines += [
        f"grXP2 {gr_xp2}", f"grYP2 {gr_yp2}", f"grPFVelInGRXPerTStep {vel}", f"grAFDelayInTStep {af_delay}",
        f"maxnumpGRfromGRtoGO {max(1, max_gr_out)}", "maxnumpGRfromGLtoGR 4", "maxnumpGRfromGOtoGR 4",
        "maxnumpGRfromMFtoGR 4", "spanGRDenOnGLX 1", "spanGRDenOnGLY 1",
        f"numSCP2 {sc_p2}", f"numPCP2 {pc_p2}", f"numpPCfromPCtoNC {pcnc}", f"numNCP2 {nc_p2}",
        f"numIOP2 {io_p2}", "connectivityParamEnd 1",
    ]
    return "\n".join(lines) + "\n"


def build_random_network(gr_xp2, gr_yp2, go_xp2, go_yp2, mf_p2, act_text, *, seed=0,
                         mf_per_gr=4, go_per_gr=3, gr_per_go=None, go_out_per_gr=None,
                         mf_per_go=16, vel=147, af_delay=1, pc_p2=5, sc_p2=9, nc_p2=3, io_p2=2,
                         pcnc=3, gogo=((0, -1, 1.0), (-1, -1, 1.0), (-1, 0, 1.0), (-1, 1, 1.0)),
                         n_zones=1, new_state=None):
    """A CBMState with random input-net wiring.

    GR->GO synapses are drawn either from the GO side (gr_per_go random GR per
    GO) or from the GR side (go_out_per_gr random GO per GR).  new_state
    (default CBMState.new) makes the empty state from the parameter texts;
    any object with the same con() / array() interface works."""
    if new_state is None:
        from . import CBMState
        new_state = CBMState.new
    rng = np.random.Generator(np.random.PCG64(seed))
    n_gr = 1 << (gr_xp2 + gr_yp2)
    gr_x = 1 << gr_xp2
    go_x, go_y = 1 << go_xp2, 1 << go_yp2
    n_go, n_mf = go_x * go_y, 1 << mf_p2

    # GR -> GO outputs
    if gr_per_go is not None:
        tg = np.stack([rng.choice(n_gr, size=gr_per_go, replace=False) for _ in range(n_go)])
        out_tab, out_cnt, max_out = _gr_lists_from_targets(tg, n_gr)
    else:
        k = go_out_per_gr or 4
        out_tab = np.sort(_distinct_choice(rng, n_gr, k, n_go), axis=1).astype(np.uint32)
        out_cnt = np.full(n_gr, k, dtype=np.int32)
        max_out = k
    # MF -> GO (per GO mf_per_go random fibres, stored MF-side)
    mg = np.stack([rng.choice(n_mf, size=mf_per_go, replace=False) for _ in range(n_go)])
    mf_go_tab, mf_go_cnt, max_mf_go = _gr_lists_from_targets(mg, n_mf)

    con = con_params_text(gr_xp2, gr_yp2, go_xp2, go_yp2, mf_p2, max_gr_out=max_out,
                          max_mf_go_per_mf=max_mf_go, vel=vel, af_delay=af_delay, sc_p2=sc_p2,
                          pc_p2=pc_p2, nc_p2=nc_p2, io_p2=io_p2, pcnc=pcnc, gogo=gogo)
    st = new_state(con, act_text, n_zones, wiring_seeds=[seed * 7 + z + 1 for z in range(n_zones)])
    max_go_stride = st.con("maxnumpGRfromGOtoGR")
    max_out_stride = st.con("maxnumpGRfromGRtoGO")
    mf_go_stride = st.con("maxnumpMFfromMFtoGO")

    # GR dendrites: MF and GO inputs; both tables have maxnumpGRfromGOtoGR columns
    mf_in = _distinct_choice(rng, n_gr, mf_per_gr, n_mf)
    go_in = _distinct_choice(rng, n_gr, go_per_gr, n_go)
    p = st.array("pGRfromMFtoGR").reshape(n_gr, max_go_stride)
    p[:, :mf_per_gr] = mf_in
    st.array("numpGRfromMFtoGR")[:] = mf_per_gr
    p = st.array("pGRfromGOtoGR").reshape(n_gr, max_go_stride)
    p[:, :go_per_gr] = go_in
    st.array("numpGRfromGOtoGR")[:] = go_per_gr

    # GR axons: targets plus delay masks (assignGRDelays)
    gr_pos_x = (np.arange(n_gr) % gr_x).astype(np.int64)
    ms_per_step = 1
    p = st.array("pGRfromGRtoGO").reshape(n_gr, max_out_stride)
    m = st.array("pGRDelayMaskfromGRtoGO").reshape(n_gr, max_out_stride)
    p[:, :out_tab.shape[1]] = out_tab
    st.array("numpGRfromGRtoGO")[:] = out_cnt
    valid = np.arange(out_tab.shape[1])[None, :] < out_cnt[:, None]
    go_of = np.where(valid, out_tab, 0).astype(np.int64)
    go_pos_x = ((go_of % go_x).astype(np.float32) * np.float32(np.float32(gr_x) / np.float32(go_x))).astype(np.int64)
    d = np.abs(go_pos_x - gr_pos_x[:, None])
    wrap = d > gr_x // 2
    d = np.where(wrap, np.where(go_pos_x < gr_pos_x[:, None], go_pos_x + gr_x - gr_pos_x[:, None],
                                gr_pos_x[:, None] + gr_x - go_pos_x), d)
    shift = (d // vel + af_delay) // ms_per_step
    m[:, :out_tab.shape[1]] = np.where(valid, (np.uint64(1) << shift.astype(np.uint64)).astype(np.uint32), 0xFFFFFFFF)
    d_bsp = np.abs(gr_x // 2 - gr_pos_x)
    st.array("pGRDelayMaskfromGRtoBSP")[:] = (1 << ((d_bsp // vel + af_delay) // ms_per_step)).astype(np.uint32)

    # MF -> GO out-lists
    p = st.array("pMFfromMFtoGO").reshape(n_mf, mf_go_stride)
    p[:, :mf_go_tab.shape[1]] = mf_go_tab[:, :mf_go_stride]
    st.array("numpMFfromMFtoGO")[:] = mf_go_cnt

    # GO -> GO from the local matrix (connectGOGO)
    out_cnt_gg = st.array("numpGOGABAOutGOGO")
    in_cnt_gg = st.array("numpGOGABAInGOGO")
    n_gg = len(gogo)
    p_out = st.array("pGOGABAOutGOGO").reshape(n_go, n_gg)
    p_in = st.array("pGOGABAInGOGO").reshape(n_go, n_gg)
    for i in range(n_go):
        cx, cy = i % go_x, i // go_x
        for (dx, dy, prob) in gogo:
            if rng.random() >= (1 - prob):
                dst = ((cy + dy) % go_y) * go_x + (cx + dx) % go_x
                p_out[i, out_cnt_gg[i]] = dst
                out_cnt_gg[i] += 1
                p_in[dst, in_cnt_gg[dst]] = i
                in_cnt_gg[dst] += 1
    return st


# ------------------------------------------------------------ configurations
def config1_network(seed=0, new_state=None):
    """16,384 GR (4 MF + 3 GO dendrites), 256 GO x 128 random GR, 1024 MF,
    32 PC x 512 PF, 128 BC, 512 SC, 8 NC, 4 IO."""
    return build_random_network(8, 6, 4, 4, 10, act_params("16k"), seed=seed, gr_per_go=128,
                                mf_per_go=3, vel=40, gogo=((1, 1, 0.0),), new_state=new_state)


def config2_network(seed=0, new_state=None):
    """1,048,576 GR (4 MF + 3 GO dendrites, 4 GO targets each), 1024 GO,
    1024 MF, 32 PC x 32,768 PF, 128 BC, 512 SC, 8 NC, 4 IO."""
    return build_random_network(11, 9, 6, 4, 10, act_params("dense"), seed=seed, go_out_per_gr=4,
                                mf_per_go=16, vel=147, new_state=new_state)


def config3_network(seed=0, new_state=None):
    """4,194,304 GR, 4096 GO x 1024 random GR, 1024 MF, 128 PC x 32,768 PF."""
    return build_random_network(12, 10, 6, 6, 10, act_params("dense"), seed=seed, gr_per_go=1024,
                                mf_per_go=16, vel=294, pc_p2=7, new_state=new_state)


class StateVariableMF:
    """Cart-pole-style MF rate coding: each of n_vars state variables owns an
    equal, ordered share of the fibres (StateVariable::assignOrderedMFInds,
    Matthew_Sim_CBM/includes/statevariable.hpp:35-43, with the unassigned
    list built from the last fibre down, environment.cpp:47-51), and the k-th
    fibre of a variable fires at a blend of its relaxed and excited rates
    weighted by a Gaussian of the distance between the variable's value and
    the fibre's preferred value (gaussMFAct, statevariable.hpp:108-129).
    rates() follows gaussMFAct's arithmetic: float values, the preferred
    values accumulated fibre by fibre from min + interval / 2, the width
    gaussWidth x interval, the Gaussian's exp and normalisation in double
    (the C library's exp, as the reference's unqualified exp on a float
    resolves to it), each rounded to float where the reference stores a
    float.  Relaxed rates are U(1, 10) Hz and excited rates 40 Hz
    (Environment::setupMossyFibers, environment.cpp:19-39, whose excited
    range expression reduces to its minimum).  gauss_width defaults to
    sigma_frac x the fibres a variable owns, a width of sigma_frac of the
    variable's range.

    The environment that moves the variables (the cart-pole dynamics) lies
    outside the simulator; values() supplies a fixed synthetic trajectory:
    variable v follows 0.5 + 0.45 sin(2 pi t / period_v + phase_v) of its
    range.
    """

    PERIODS = (1000.0, 1700.0, 2300.0, 3100.0)

    def __init__(self, num_mf, seed=0, n_vars=4, sigma_frac=0.2, lo=-1.0, hi=1.0, gauss_width=None):
        f32 = np.float32
        rng = np.random.Generator(np.random.PCG64(seed + 303))
        self.num_mf = num_mf
        self.n_vars = n_vars
        self.lo, self.hi = f32(lo), f32(hi)
        self.relaxed = rng.uniform(1.0, 10.0, num_mf).astype(np.float32)
        self.excited = np.full(num_mf, 40.0, dtype=np.float32)
        self.phase = rng.uniform(0, 2 * np.pi, n_vars)
        # StateVariable::initialize: numMF = totalMF * mfProportion, a float product truncated
        per = int(f32(num_mf) * (f32(1) / f32(n_vars)))
        self.per = per
        self.gauss_width = f32(sigma_frac * per) if gauss_width is None else f32(gauss_width)
        self.interval = f32(f32(self.hi - self.lo) / f32(per))
        # preferred values: pos = min + interval / 2.0 (a double sum stored as float), then pos += interval
        pos = f32(float(self.lo) + float(self.interval) / 2.0)
        means = np.zeros(per, np.float32)
        for k in range(per):
            means[k] = pos
            pos = f32(pos + self.interval)
        self.var_of = np.full(num_mf, -1, dtype=np.int64)
        self.mean = np.zeros(num_mf, dtype=np.float32)
        for v in range(n_vars):
            self.var_of[v * per: (v + 1) * per] = v
            self.mean[v * per: (v + 1) * per] = means
        self.variance = f32(self.gauss_width * self.interval)  # the reference's name for the width
        var2 = f32(self.variance * self.variance)
        self._den = f32(f32(2) * var2)
        self._norm = math.sqrt(2 * math.pi * float(var2))
        self._max_possible = f32(1.0 / self._norm)

    def values(self, t):
        """The n_vars state-variable values at step t (synthetic trajectory)."""
        ph = 2 * np.pi * t / np.array(self.PERIODS[: self.n_vars]) + self.phase
        return (self.lo + (self.hi - self.lo) * (0.5 + 0.45 * np.sin(ph))).astype(np.float32)

    def rates_for(self, x):
        """[num_mf] Hz for state values x [n_vars] (gaussMFAct for every
        variable); fibres beyond the variables' shares stay relaxed."""
        f32 = np.float32
        out = self.relaxed.copy()
        m = self.var_of >= 0
        x = np.asarray(x, dtype=np.float32)
        xv = np.maximum(self.lo, np.minimum(self.hi, x))[self.var_of[m]]
        d = (xv - self.mean[m]).astype(np.float32)
        arg = ((-(d * d)).astype(np.float32) / self._den).astype(np.float32)
        value = (np.array([math.exp(a) for a in arg.astype(np.float64)]) / self._norm).astype(np.float32)
        a = (value / self._max_possible).astype(np.float32)
        out[m] = ((a * self.excited[m]).astype(np.float32) +
                  ((f32(1) - a).astype(np.float32) * self.relaxed[m]).astype(np.float32)).astype(np.float32)
        return out

    def rates(self, t):
        """[num_mf] Hz at step t of the synthetic trajectory."""
        return self.rates_for(self.values(t))

    def trajectory(self, steps):
        """The synthetic trajectory's values for steps 1..steps, [steps,
        n_vars]: the rows a device state-variable input takes step by step
        (CBMSimCore.set_statevar_input)."""
        return np.stack([self.values(t) for t in range(1, steps + 1)]).astype(np.float32)


def config3_mf_stream(num_mf, steps, seed=0):
    """MF spikes of the dense 4M configuration: regenerating Poisson fibres
    driven by the state-variable rate coding."""
    coding = StateVariableMF(num_mf, seed=seed)
    gen = RegenPoissonMF(num_mf, seed)
    return gen.run(coding.rates, steps)


def eyelid_mf_rates(num_mf, seed=0, cs_count=80):
    """Config-2 MF rates: 10% tonic at U(50,80) Hz, the rest U(1,10) Hz; the
    first cs_count fibres of a random permutation carry the CS (100 Hz)."""
    rng = np.random.Generator(np.random.PCG64(seed + 101))
    bg = rng.uniform(1, 10, num_mf).astype(np.float32)
    tonic = rng.random(num_mf) < 0.1
    bg[tonic] = rng.uniform(50, 80, int(tonic.sum())).astype(np.float32)
    cs = rng.permutation(num_mf)[:cs_count]
    cs_rates = bg.copy()
    cs_rates[cs] = np.float32(100.0)
    return bg, cs_rates


def eyelid_mf_stream(num_mf, steps, seed=0, cs_on=2000, cs_off=2500, trial_len=5000):
    """MF spikes of the eyelid protocol: CS rates inside [cs_on, cs_off) of each trial."""
    bg, cs = eyelid_mf_rates(num_mf, seed)
    gen = RegenPoissonMF(num_mf, seed)

    def freqs(t):
        tt = (t - 1) % trial_len
        return cs if cs_on <= tt < cs_off else bg
    return gen.run(freqs, steps)


def uniform_mf_stream(num_mf, steps, seed=0, lo=1.0, hi=30.0):
    """MF spikes with fixed rates drawn U(lo, hi) Hz (config 1)."""
    rng = np.random.Generator(np.random.PCG64(seed + 202))
    rates = rng.uniform(lo, hi, num_mf).astype(np.float32)
    gen = RegenPoissonMF(num_mf, seed)
    return gen.run(lambda t: rates, steps)


class MFPopulation:
    """MF rate tables of an eyelid protocol in the reference's ECMFPopulation
    form (CBM_TOOLS_LIB_DEV/src/ecmfpopulation.cpp): background, CS-tonic and
    CS-phasic Hz per fibre.  ``rates()`` is what set_eyelid_protocol takes.

    Tables the reference's tools library generates can be read from its file
    (``read``; writeToFile's layout: i32 numMF, then the three f32 tables), and
    ``from_trial_data`` re-estimates the tables from a recorded MF histogram
    as the reference's ECMFPopulation(ECTrialsData *) does."""

    def __init__(self, bg, cs_tonic, cs_phasic):
        self.bg = np.ascontiguousarray(bg, dtype=np.float32)
        self.cs_tonic = np.ascontiguousarray(cs_tonic, dtype=np.float32)
        self.cs_phasic = np.ascontiguousarray(cs_phasic, dtype=np.float32)

    def rates(self):
        """[3, numMF] Hz: background, CS tonic, CS phasic."""
        return np.stack([self.bg, self.cs_tonic, self.cs_phasic])

    @classmethod
    def random(cls, num_mf, seed, frac_cs_tonic, frac_cs_phasic, frac_context,
               bg_min, cs_bg_min, context_min, cs_tonic_min, cs_phasic_min,
               bg_max, cs_bg_max, context_max, cs_tonic_max, cs_phasic_max):
        """ECMFPopulation(numMF, randSeed, fracCSTMF, ...) (ecmfpopulation.cpp:
        67-190), the parameters in its order: every fibre starts at a uniform
        background rate; distinct CS-tonic, then CS-phasic, then context
        fibres are picked (int(frac x numMF) of each, in float as the
        reference counts them); context fibres get one context rate for all
        three tables, CS fibres a CS-background rate plus a CS-tonic
        (tonic fibres, used in both CS tables) or CS-phasic rate (phasic
        fibres, phasic table only).  The draws come from the package's
        generator, not the reference's SFMT stream, which the eyelid driver
        seeds with the wall clock (mainw.cpp:208)."""
        f32 = np.float32
        rng = np.random.Generator(np.random.PCG64(seed + 404))

        def u(lo, hi, n):
            return (rng.random(n) * (f32(hi) - f32(lo)) + f32(lo)).astype(np.float32)
        bg = u(bg_min, bg_max, num_mf)
        tonic, phasic = bg.copy(), bg.copy()
        n_t, n_p, n_c = (int(f32(f) * f32(num_mf)) for f in (frac_cs_tonic, frac_cs_phasic, frac_context))
        if n_t + n_p + n_c > num_mf:
            raise ValueError("the CS-tonic, CS-phasic and context fractions add up to more than every fibre")
        order = rng.permutation(num_mf)
        t_idx, p_idx, c_idx = order[:n_t], order[n_t: n_t + n_p], order[n_t + n_p: n_t + n_p + n_c]
        bg[c_idx] = u(context_min, context_max, n_c)
        tonic[c_idx] = phasic[c_idx] = bg[c_idx]
        bg[t_idx] = u(cs_bg_min, cs_bg_max, n_t)
        tonic[t_idx] = phasic[t_idx] = u(cs_tonic_min, cs_tonic_max, n_t)
        bg[p_idx] = tonic[p_idx] = u(cs_bg_min, cs_bg_max, n_p)
        phasic[p_idx] = u(cs_phasic_min, cs_phasic_max, n_p)
        return cls(bg, tonic, phasic)

    @classmethod
    def read(cls, path):
        """ECMFPopulation(fstream &) (ecmfpopulation.cpp:192-211)."""
        with open(path, "rb") as f:
            n = int(np.frombuffer(f.read(4), np.int32)[0])
            t = np.frombuffer(f.read(12 * n), np.float32)
        if t.size != 3 * n:
            raise ValueError(f"{path}: truncated MF population file")
        return cls(t[:n], t[n: 2 * n], t[2 * n:])

    def write(self, path):
        """ECMFPopulation::writeToFile (ecmfpopulation.cpp:220-235)."""
        with open(path, "wb") as f:
            f.write(np.int32(self.bg.size).tobytes())
            for a in (self.bg, self.cs_tonic, self.cs_phasic):
                f.write(a.tobytes())

    @classmethod
    def from_trial_data(cls, mf_psh, num_trials, bin_steps, pre_cs, cs_ms):
        """ECMFPopulation(ECTrialsData *) (ecmfpopulation.cpp:11-65) from the
        MF histogram f32 [bins][numMF] of num_trials recorded trials, binned
        by bin_steps, with pre_cs ms before the CS and a CS of cs_ms: the mean
        rate over the background bins [2, preBins - 2), the CS-phasic bins
        [preBins + 1, preBins + 3) and the CS-tonic bins
        [preBins + csBins - 6, preBins + csBins - 1), in float as the
        reference sums them (bin by bin, then one divide).  As in the
        reference, the bin width counts as milliseconds."""
        f32 = np.float32
        # float scaling = numTrials * (msPerBin / 1000.0): a double product stored as float
        scaling = f32(num_trials * (bin_steps / 1000.0))
        pre_bins, cs_bins = pre_cs // bin_steps, cs_ms // bin_steps
        psh = np.asarray(mf_psh, dtype=np.float32)

        def mean(lo, hi, count):
            s = np.zeros(psh.shape[1], np.float32)
            for j in range(lo, hi):
                s = (s + psh[j]).astype(np.float32)
            return (s / (f32(count) * scaling)).astype(np.float32)
        return cls(mean(2, pre_bins - 2, pre_bins - 4), mean(pre_bins + cs_bins - 6, pre_bins + cs_bins - 1, 5),
                   mean(pre_bins + 1, pre_bins + 3, 2))
