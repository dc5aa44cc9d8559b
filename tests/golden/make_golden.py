"""Regenerates the golden fixtures of tests/golden from the reference itself.

Runs here, where the reference tree and its harness (oracle/_ref, built by
`make -C oracle ref`) exist:
  ref16k.state.xz        a 16,384-GR network built by the reference's own
                         generator from CBM_Params/actParams_16K_Gr.txt and
                         conParams_16K_Gr.txt (oracle/_ref/ref_gen, seeds 11/22/33)
  ref16k_digests.json    SHA-256 of every trace record of the reference's
                         calcActivity over 1500 steps of a fixed MF input with
                         plasticity, error-drive and GR->GO gain events, plus
                         the SHA-256 of the final state file
  config1_digests.json   the same for the synthetic 16K network of the package
                         (config 1), built with networks.config1_network(seed=0)
  config2_digests.json   the same for the 1M-GR network (networks.config2_network,
                         1000 steps of eyelid-coded MF input with a CS,
                         plasticity that moves PF->PC weights, and error
                         drives), plus the SHA-256 of every array of the
                         initial and final states
  config3_digests.json   the same for the dense 4M-GR network
                         (networks.config3_network, 400 steps of state-variable
                         coded MF input)
  (the inputs of both: cbmtest.golden_large_case)

usage: python tests/golden/make_golden.py [/path/to/reference]
"""
import json
import lzma
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

import cbmtest  # noqa: E402

EVENTS16K = {
    5: [("plast", 0, -0.01, 0.005)],
    700: [("errdrive", 0, 1.0)],
    1000: [("errdrive", 0, 0.6)],
    1200: [("plastreset", 0)],
    1300: [("grgoinc", 0.01)],
    1400: [("grgoincreset",)],
}
STEPS16K = 1500
MF_SEED16K = 11
ZONE_SEEDS = [7]


def digests(trace, rb, final_state):
    tr = trace.reshape(-1, rb)
    with open(final_state, "rb") as f:
        fin = f.read()
    return {"record_bytes": int(rb), "steps": int(tr.shape[0]),
            "records": [cbmtest.sha(r) for r in tr], "final_state": cbmtest.sha(np.frombuffer(fin, np.uint8))}


def main(ref_root):
    with tempfile.TemporaryDirectory() as d:
        st = os.path.join(d, "ref16k.state")
        params = os.path.join(ref_root, "CBM_Params")
        subprocess.run([cbmtest.REF_GEN, os.path.join(params, "actParams_16K_Gr.txt"),
                        os.path.join(params, "conParams_16K_Gr.txt"), "1", "11", "22", "33", st],
                       check=True, capture_output=True)
        with open(st, "rb") as f, lzma.open(os.path.join(HERE, "ref16k.state.xz"), "wb", preset=9) as g:
            g.write(f.read())
        mf = cbmtest.counter_mf(1024, STEPS16K, MF_SEED16K)
        fin = os.path.join(d, "final.state")
        tr = cbmtest.ref_run(st, mf, ZONE_SEEDS, EVENTS16K, final_path=fin)
        rb = tr.size // STEPS16K
        with open(os.path.join(HERE, "ref16k_digests.json"), "w") as f:
            json.dump(digests(tr, rb, fin), f)

        from cerebellum_simulation_b200 import networks
        net = networks.config1_network(seed=0)
        p1 = os.path.join(d, "config1.state")
        net.writeState(p1)
        mf1 = networks.uniform_mf_stream(1024, 1000, seed=0)
        fin1 = os.path.join(d, "final1.state")
        tr1 = cbmtest.ref_run(p1, mf1, ZONE_SEEDS, None, final_path=fin1)
        out = digests(tr1, tr1.size // 1000, fin1)
        with open(p1, "rb") as f:
            out["initial_state"] = cbmtest.sha(np.frombuffer(f.read(), np.uint8))
        with open(os.path.join(HERE, "config1_digests.json"), "w") as f:
            json.dump(out, f)

        for name in ("config2", "config3"):
            net, mf, events = cbmtest.golden_large_case(name)
            steps = mf.shape[0]
            p = os.path.join(d, name + ".state")
            net.writeState(p)
            del net
            fin = os.path.join(d, name + "_final.state")
            tr = cbmtest.ref_run(p, mf, ZONE_SEEDS, events, final_path=fin)
            out = digests(tr, tr.size // steps, fin)
            del tr
            with open(p, "rb") as f:
                out["initial_state"] = cbmtest.sha(np.frombuffer(f.read(), np.uint8))
            out["initial_arrays"] = cbmtest.state_array_digests(p)
            out["final_arrays"] = cbmtest.state_array_digests(fin)
            with open(os.path.join(HERE, name + "_digests.json"), "w") as f:
                json.dump(out, f)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
