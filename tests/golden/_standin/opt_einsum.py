"""Minimal stand-in for the third-party ``opt_einsum`` package (pinned by the
reference as ``opt-einsum>=3.4.0``, absent from this image).

Only ``tests/golden/make_goldens.py`` puts this directory on ``sys.path``, so
that the reference's own ``CCM/coupled_cluster.py`` and ``CCM/ccDgrams.py``
(which do ``from opt_einsum import contract``) can be imported to produce the
golden vectors.  ``contract`` is a tensor contraction; numpy's einsum computes
the same sums, only the FP64 summation order differs.
"""
import numpy as np


def contract(subscripts, *operands, optimize="greedy", **kwargs):
    if optimize is True or optimize is None:
        optimize = "greedy"
    return np.einsum(subscripts, *operands, optimize=optimize)


def contract_path(subscripts, *operands, **kwargs):
    return np.einsum_path(subscripts, *operands, optimize="greedy")
