"""Load a golden fixture written by make_golden.py into (Net, inputs, ref)."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ("cfg1", "cfg2", "cfg2_wide", "feat_mid", "feat_low", "cfg3_small", "cfg3_tcv")


def load(tag):
    from wdsgpu_b200.net import Net
    z = np.load(os.path.join(HERE, tag + ".npz"))
    fields = {}
    for k in z.files:
        if not k.startswith("net__"):
            continue
        name = k[5:]
        v = z[k]
        if name in ("node_id", "link_id", "pattern_ids", "meta", "controls_raw",
                    "rules_raw"):
            v = json.loads(str(v))
        elif name == "patterns":
            v = [np.asarray(p) for p in json.loads(str(v))]
        fields[name] = v
    net = Net(**fields)
    inp = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    ref = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    return net, inp, ref
