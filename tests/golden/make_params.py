"""Regenerates the activity-parameter sets shipped with the package.

The model constants (leak conductances, decay times, thresholds, plasticity
steps) are the reference's; they define the network being simulated, so the
bundled sets are taken from the reference's parameter files
(CBM_Params/actParams_16K_Gr.txt and CBM_Params/actParams_dense_4MGR_dev.txt)
and written in the key/value form ActivityParams(fstream&) reads
(CBM_STATE_LIB_DEV/src/params/activityparams.cpp:12-42).

Test-side tooling: it reads the reference tree, so it lives beside the golden
fixtures' generator and writes into cerebellum_simulation_b200/params/.

usage: python tests/golden/make_params.py /path/to/reference/CBM_Params
"""
import os
import sys

SETS = {"act_16k.txt": "actParams_16K_Gr.txt", "act_dense.txt": "actParams_dense_4MGR_dev.txt"}
# connectivity sets, copied line by line up to their end marker (the GO-GO
# matrix block has rows of three values)
CON_SETS = {"con_16k.txt": "conParams_16K_Gr.txt"}


def convert_con(src, dst):
    out = []
    with open(src) as f:
        for line in f:
            line = " ".join(line.split())
            if not line:
                continue
            out.append(line)
            if line.startswith("connectivityParamEnd"):
                break
    with open(dst, "w") as f:
        f.write("\n".join(out) + "\n")


def convert(src, dst):
    pairs = []
    with open(src) as f:
        toks = f.read().split()
    for k, v in zip(toks[0::2], toks[1::2]):
        if k == "activityParamEnd":
            break
        pairs.append((k, v))
    with open(dst, "w") as f:
        for k, v in pairs:
            f.write(f"{k} {v}\n")
        f.write("activityParamEnd 1\n")


if __name__ == "__main__":
    ref = sys.argv[1]
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    dest = os.path.join(root, "cerebellum_simulation_b200", "params")
    for out, src in SETS.items():
        convert(os.path.join(ref, src), os.path.join(dest, out))
        print(out)
    for out, src in CON_SETS.items():
        convert_con(os.path.join(ref, src), os.path.join(dest, out))
        print(out)
