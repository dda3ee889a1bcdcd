"""Conserved totals of a case's register, summed exactly.

A total over millions of nearly equal cells summed in floating point carries
an error of the order of the cell count times the rounding unit, and that
error changes with the cells' last bits: numpy's sum over the 128^3
Taylor-Green field moves by 1e-12 of the mass between two states whose
exact totals are equal to the bit.  math.fsum sums exactly (then rounds
once), so a conservation bar reads the solver's arithmetic alone.
"""

import math

import numpy as np


def totals(mb, reg="Q"):
    """Each component's total of volume times the interior cells' values,
    over every block, summed exactly."""
    parts = None
    for b, m in zip(mb.blocks, mb.metrics):
        vol = 1.0 / m["detJinv"][b.mesh.interior]
        q = getattr(b, reg).get()[b.mesh.interior]
        prods = [(q[..., c] * vol).ravel() for c in range(q.shape[-1])]
        if parts is None:
            parts = [[] for _ in prods]
        for acc, p in zip(parts, prods):
            acc.append(math.fsum(p))
    return np.array([math.fsum(a) for a in parts])
