"""Surrogate-proposed parameter sweeps of the eyelid-conditioning network.

A sweep asks which parameter sets give the largest conditioned response.  The
plain way simulates every candidate.  Here the batched simulator
(:class:`CBMBatch`, device-driven trials) generates training trials, the
surrogate MLP (:mod:`.surrogate`, tensor-core kernels) learns the trial's
50-bin NC rate trace from a 64-value description of the parameters and the
MF input, ranks all candidates, and only the best ones are simulated in full;
the simulator stays the arbiter of the surrogate's error.

Parameters of a set (each drawn uniformly, scales log-uniformly):
  GO threshold scale 0.8-1.2, PF->PC LTD and LTP step scales 0.5-2,
  MF background-rate scale 0.5-1.5, CS MF rate 40-120 Hz, GR->GO gain scale
  0.5-1.5, and the seed of the MF rate table and generator.
"""
import numpy as np

from . import CBMBatch, CBMState, eyelid_protocol_defaults

N_PARAMS = 6
N_FEATURES = 64
N_TRACE = 50

# trials of the sweep: CS 500-1000 of 1500-step trials, recorded over the
# whole trial in 10-step bins, NC rate trace in 50 bins of 30 steps
TRIAL = dict(trialSteps=1500, csOn=500, csOff=1000, csPhasicOff=500, csStartTrial=0, preCS=500, postCS=500,
             binSteps=10, plastOnDelay=200, plastOffDelay=200)
LO = np.array([0.8, 0.5, 0.5, 0.5, 40.0, 0.5])
HI = np.array([1.2, 2.0, 2.0, 1.5, 120.0, 1.5])
LOG = np.array([False, True, True, False, False, False])


def draw_params(n, seed):
    """n parameter sets [n, 6] and MF seeds [n]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = rng.uniform(0, 1, (n, N_PARAMS))
    p = np.where(LOG, np.exp(np.log(LO) + u * (np.log(HI) - np.log(LO))), LO + u * (HI - LO))
    return p, rng.integers(1, 2**31 - 1, n)


def mf_rates(num_mf, params, mf_seed):
    """[3, num_mf] Hz: background U(1,30) x scale, CS on a random 10%."""
    rng = np.random.Generator(np.random.PCG64(int(mf_seed)))
    bg = (rng.uniform(1.0, 30.0, num_mf) * params[3]).astype(np.float32)
    cs = bg.copy()
    cs[rng.permutation(num_mf)[: num_mf // 10]] = params[4]
    return np.stack([bg, cs, cs]).astype(np.float32)


def features(params, mf_seeds, trial, trials, nc_inputs, num_mf=1024):
    """[n, 64]: the six parameters scaled to [-1, 1], the trial index, and the
    MF input pattern of num_mf fibres: the mean background and CS-phase rate
    of each NC's MF inputs (nc_inputs: [numNC, inputs] MF indices of zone 0,
    at most 8 NCs), then quantiles of all background and CS-phase rates
    (Hz / 100)."""
    n = params.shape[0]
    num_nc = nc_inputs.shape[0]
    out = np.zeros((n, N_FEATURES), dtype=np.float32)
    x = np.where(LOG, (np.log(params) - np.log(LO)) / (np.log(HI) - np.log(LO)), (params - LO) / (HI - LO))
    out[:, :N_PARAMS] = 2 * x - 1
    out[:, N_PARAMS] = 2 * np.asarray(trial, dtype=np.float32) / max(1, trials - 1) - 1
    k = N_PARAMS + 1
    nq = (N_FEATURES - k - 2 * min(num_nc, 8)) // 2
    qb, qc = np.linspace(0, 1, nq), np.linspace(0, 1, N_FEATURES - k - 2 * min(num_nc, 8) - nq)
    for i in range(n):
        r = mf_rates(num_mf, params[i], mf_seeds[i])
        j = k
        for c in range(2):
            m = r[c][nc_inputs[:8]].mean(1) / 100
            out[i, j:j + len(m)] = m
            j += len(m)
        out[i, j:j + nq] = np.quantile(r[0], qb) / 100
        j += nq
        out[i, j:N_FEATURES] = np.quantile(r[1], qc) / 100
    return out


def nc_inputs_of(state):
    """[numNC, inputs] MF indices of zone 0's NCs (pNCfromMFtoNC)."""
    return state.array("pNCfromMFtoNC", 0).reshape(state.con("numNC"), -1).astype(np.int64)


def nc_trace(nc_psh, num_nc):
    """[trials, bins, numNC] counts per 10-step bin -> [trials, 50] NC rate (Hz)."""
    c = nc_psh.sum(axis=2).astype(np.float64)
    c = c[:, : (c.shape[1] // 3) * 3].reshape(c.shape[0], -1, 3).sum(axis=2)
    return (c / (num_nc * 0.030)).astype(np.float32)


def pc_trace(pc_psh, num_pc):
    """[trials, bins, numPC] counts per 10-step bin -> [trials, 50] mean PC
    rate (Hz), binned as nc_trace."""
    return nc_trace(pc_psh, num_pc)


def trace_rmse_over_range(pred, truth):
    """Root-mean-square error of predicted traces over the range of the true
    traces (max - min over all of them): the sweep's error measure."""
    pred, truth = np.asarray(pred, np.float64), np.asarray(truth, np.float64)
    span = float(truth.max() - truth.min())
    return float(np.sqrt(np.mean((pred - truth) ** 2))) / max(span, 1e-9)


def objective(traces):
    """Conditioned response of a trace (or [.., 50] traces): mean NC rate over
    the late CS (steps 800-1000) minus the pre-CS mean (steps 0-500)."""
    t = np.asarray(traces)
    return t[..., 27:33].mean(-1) - t[..., 0:16].mean(-1)


def simulate(base_state, params, mf_seeds, trials, device=0, batch=256, chunk=250):
    """Trials of every parameter set through the batched simulator:
    [n, trials, 50] NC rate traces and the seconds of device time."""
    traces, secs = simulate_traces(base_state, params, mf_seeds, trials, device, batch, chunk)
    return traces["nc"], secs


def simulate_traces(base_state, params, mf_seeds, trials, device=0, batch=256, chunk=250):
    """As simulate, with both responses: ({"nc": [n, trials, 50] NC rate
    traces, "pc": [n, trials, 50] mean PC rate traces}, device seconds)."""
    out, out_pc, gpu_ms = [], [], 0.0
    for b0 in range(0, params.shape[0], batch):
        idx = range(b0, min(params.shape[0], b0 + batch))
        states = []
        for i in idx:
            st = CBMState(base_state)
            st.setActParam("threshBaseGO", st.act("threshBaseGO") * params[i, 0])
            st.setActParam("gGRIncGO", st.act("gGRIncGO") * params[i, 5])
            states.append(st)
        b = CBMBatch(states, [[11 + i] for i in idx], device=device)
        for k, i in enumerate(idx):
            st = states[k]
            proto = eyelid_protocol_defaults(st, mfSeed=int(mf_seeds[i]) & 0x7FFFFFFF, numDataTrials=trials,
                                             dataStartTrial=0, **TRIAL)
            proto["plastLTD"] *= params[i, 1]
            proto["plastLTP"] *= params[i, 2]
            b.set_eyelid_protocol(k, mf_rates(st.con("numMF"), params[i], mf_seeds[i]), **proto)
        steps = trials * TRIAL["trialSteps"]
        gpu_ms += b.run(steps, chunk)
        for k, i in enumerate(idx):
            out.append(nc_trace(b.trial_record(k, "nc"), states[k].con("numNC")))
            out_pc.append(pc_trace(b.trial_record(k, "pc"), states[k].con("numPC")))
        b.close()
    return {"nc": np.stack(out), "pc": np.stack(out_pc)}, gpu_ms / 1000.0


def fit_surrogate(net, x, traces, epochs=150, lr=1e-3, seed=0):
    """Train net on log(1 + rate) of the traces; returns the last epoch's loss."""
    return net.train(x, np.log1p(traces).astype(np.float32), batch=min(256, net.max_batch), epochs=epochs, lr=lr,
                     seed=seed)


def predict(net, x):
    """NC rate traces (Hz) the surrogate predicts for feature rows x."""
    return np.maximum(np.expm1(net.forward(x)), 0.0)
