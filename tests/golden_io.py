"""Load the golden fixtures written by tests/golden/make_goldens.py."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def dense(g, name):
    out = np.zeros(tuple(g[name + "_shape"]))
    idx = g[name + "_idx"]
    if len(idx):
        out[tuple(idx.T)] = g[name + "_val"]
    return out


def rows(g, name):
    """[k0,k1,k2,k3,val] rows of a sparse list block."""
    idx, val = g[name + "_idx"], g[name + "_val"]
    return np.concatenate([idx.astype(np.float64), val[:, None]], axis=1) if len(val) else np.zeros((0, 5))


def hamiltonian(g):
    """(fock_mats, two_body_int) in the reference's sparse=True calling form."""
    fock = [g["f_pp"], g["f_ph"], g["f_hh"]]
    two = [rows(g, "v_pppp"), rows(g, "v_ppph"), dense(g, "v_pphh"), dense(g, "v_phph"),
           dense(g, "v_phhh"), dense(g, "v_hhhh")]
    return fock, two
