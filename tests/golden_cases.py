"""Test helper: load the golden fixtures and rebuild their inputs."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

NAMES = sorted(make_golden.CASES)


def load(name):
    i = NAMES.index(name)
    case = make_golden.CASES[name]
    a1, a2, rhs = make_golden.inputs(case, i)
    G = dict(np.load(os.path.join(HERE, "golden", name + ".npz")))
    return case, a1, a2, rhs, G


def unflatten(G, key):
    data, ptr = G[key], G[key + "_ptr"] if key + "_ptr" in G else None
    return [data[ptr[k]:ptr[k + 1]] for k in range(len(ptr) - 1)]
