"""Substrates made by the reference's own generator (3DgrainMPI/graph_datastruct.py,
graph(lxd, seed), :194-271) for the forcing-folder format test.

graph_datastruct imports matplotlib at import time for its plotting helpers
(:13-21); matplotlib is not installed here, so those names are stubbed before the
import (nothing on the substrate path uses them: the map is rasterised with PIL,
the cells come from scipy's Voronoi).  Each output holds alpha (the
(nx+1) x (ny+1) map input_file.py:141-148 saves as alpha.txt), theta
([0, theta_x[1..NG], theta_z[1..NG]], input_file.py:145) and NG.

Needs the reference tree; run once, the .npz files are committed:
    python tests/golden/substrate/make_graph_substrate.py /path/to/reference
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [(20.48, 1), (20.48, 7)]  # (lxd in um, seed): 257 x 257 pixel maps


def stub_matplotlib():
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    cm = types.ModuleType("matplotlib.cm")
    colors = types.ModuleType("matplotlib.colors")
    plt.rcParams = {}
    cm.get_cmap = lambda name, n=None: (lambda x: np.zeros((len(x), 4)))
    colors.ListedColormap = lambda c: c
    mpl.pyplot, mpl.cm, mpl.colors = plt, cm, colors
    sys.modules.update({"matplotlib": mpl, "matplotlib.pyplot": plt, "matplotlib.cm": cm,
                        "matplotlib.colors": colors})


def main(reference):
    stub_matplotlib()
    sys.path.insert(0, os.path.join(reference, "3DgrainMPI"))
    from graph_datastruct import graph
    for lxd, seed in CASES:
        g = graph(lxd=lxd, seed=seed)
        alpha = np.asarray(g.alpha_field)
        ng = len(g.regions)
        theta = np.hstack([0, g.theta_x[1:], g.theta_z[1:]])
        assert alpha.min() >= 1 and alpha.max() <= ng
        out = os.path.join(HERE, "graph_lxd%g_seed%d.npz" % (lxd, seed))
        np.savez_compressed(out, alpha=alpha.astype(np.int16), theta=theta.astype(np.float64),
                            ng=np.int64(ng), lxd=np.float64(lxd), seed=np.int64(seed))
        print(out, alpha.shape, ng)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CUPF_REFERENCE", "/root/reference"))
