"""Shared helpers of the test suite."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = json.loads(str(z["config"]))
    return kw, {k: z[k] for k in z.files if k != "config"}


class Cfg:
    """Attribute bag with the reference Config fields (plus derived Nt, dx, dy)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)
        self.Nz = kw.get("Nz", 0)
        self.Lz = kw.get("Lz", 0.0)
