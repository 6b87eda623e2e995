"""General (dense) CCSD engine -- see ccsd.ccsd_solver."""


def solve(*args, **kwargs):
    raise NotImplementedError("general dense engine not built yet")
