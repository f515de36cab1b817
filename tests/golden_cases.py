"""Loader for the reference-generated fixtures in tests/golden (see make_golden.py)."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TREE_KEYS = ["key", "ni", "nx", "leafs", "nonleafs", "src_perm", "trg_perm", "colleagues", "m2l",
             "p2p_off", "p2p", "m2p_off", "m2p", "p2l_off", "p2l"]


def case_names():
    return sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(f).startswith(("p2p_", "f32ref_")))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["kernel"] = str(d["kernel"])
    d["wavek"] = complex(d["wavek"])
    d["p"] = int(d["p"])
    d["ncrit"] = int(d["ncrit"])
    d["depth_arg"] = int(d["depth_arg"])
    d["nonadaptive_depth"] = None if d["depth_arg"] < 0 else d["depth_arg"]
    d["tree"] = {k: d["tree_" + k] for k in TREE_KEYS}
    d["tree"]["depth"] = int(d["tree_depth"])
    d["tree"]["r0"] = float(d["tree_r0"])
    return d


def load_f32ref(name):
    """A fixture of the reference's single-precision build (make_golden.py main_f32)."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["kernel"] = str(d["kernel"])
    d["wavek"] = complex(d["wavek"])
    d["p"], d["ncrit"] = int(d["p"]), int(d["ncrit"])
    return d


def load_p2p():
    z = np.load(os.path.join(GOLDEN, "p2p_kernels.npz"))
    return {k: z[k] for k in z.files}
