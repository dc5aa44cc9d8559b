"""Surrogate-proposed sweep (cerebellum_simulation_b200.sweep): the MLP trained
on trials of the batched simulator predicts held-out NC rate traces better
than the method without it (predicting the mean training trace, judged by
the median absolute error: most parameter sets leave the NCs silent and a
few make them fire strongly), and the candidates it ranks highest have, when
simulated in full, a larger conditioned response than candidates drawn at
random."""
import numpy as np
import pytest

import cbmtest

pytestmark = pytest.mark.gpu

TRIALS = 4


def test_surrogate_beats_mean_trace_and_random_picks(tmp_path):
    import cerebellum_simulation_b200 as cbm
    from cerebellum_simulation_b200 import sweep
    from cerebellum_simulation_b200.surrogate import MLP
    base = cbmtest.golden_state("ref16k", str(tmp_path))
    conn = sweep.nc_inputs_of(cbm.CBMState(base))
    p_tr, s_tr = sweep.draw_params(640, seed=1)
    traces, _ = sweep.simulate(base, p_tr, s_tr, TRIALS)          # [640, 4, 50]
    n_tr = 512
    # trials after the first (its start-up transient is not part of the sweep)
    x = np.concatenate([sweep.features(p_tr[:n_tr], s_tr[:n_tr], [k] * n_tr, TRIALS, conn) for k in range(1, TRIALS)])
    t = np.concatenate([traces[:n_tr, k] for k in range(1, TRIALS)])
    net = MLP(sweep.N_FEATURES, 256, 256, sweep.N_TRACE, max_batch=256, seed=3)
    sweep.fit_surrogate(net, x, t, epochs=200, lr=1e-3, seed=4)
    # held-out instances, last trial
    x_te = sweep.features(p_tr[n_tr:], s_tr[n_tr:], [TRIALS - 1] * (640 - n_tr), TRIALS, conn)
    y_te = traces[n_tr:, TRIALS - 1]
    pred = sweep.predict(net, x_te)
    mae = float(np.median(np.abs(pred - y_te)))
    mae_mean = float(np.median(np.abs(traces[:n_tr, TRIALS - 1].mean(0) - y_te)))
    assert mae < 0.5 * mae_mean, (mae, mae_mean)
    # ranking: top 48 of 1024 candidates by predicted response vs 48 at random
    p_c, s_c = sweep.draw_params(1024, seed=7)
    pred_c = sweep.predict(net, sweep.features(p_c, s_c, [TRIALS - 1] * 1024, TRIALS, conn))
    top = np.argsort(-sweep.objective(pred_c))[:48]
    rnd = np.random.Generator(np.random.PCG64(9)).permutation(1024)[:48]
    sim_top, _ = sweep.simulate(base, p_c[top], s_c[top], TRIALS)
    sim_rnd, _ = sweep.simulate(base, p_c[rnd], s_c[rnd], TRIALS)
    j_top = sweep.objective(sim_top[:, TRIALS - 1]).mean()
    j_rnd = sweep.objective(sim_rnd[:, TRIALS - 1]).mean()
    assert j_top > j_rnd, (j_top, j_rnd)
