"""Starting branch lengths for the irreversible edit model from the
reference's parsimony change counts.

The reference gives each edge the number of characters that change along it
(charAncestralEC, src/functions.cpp:3085-3150; R stores them as the edge
lengths in collapse.infoless, R/CasPhy_functions.R:834-845).  Under the
irreversible model an unedited site leaves state 0 along an edge of time t with
probability 1 - exp(-rate t), so k edits among the parent's n0 unedited sites
give t = -log(1 - k / n0) / rate, the maximum-likelihood time of that edge alone.
Starting L-BFGS there instead of at one constant length puts every edge near its
scale, from the parsimony pass the reference already runs.
"""
from __future__ import annotations

import numpy as np

T_MIN, T_MAX = 1e-6, 10.0


def parsimony_start(edge, node_states, changes, ntip: int, rate: float = 1.0,
                    max_fraction: float = 0.95) -> np.ndarray:
    """Per-edge starting times.

    edge:        (nedge, 2) parent, child (0-based; parents are internal nodes >= ntip)
    node_states: (nnode, nsite) internal-node states from `lib.ancestral_char`
                 (row = node - ntip; 0 = unedited)
    changes:     (nedge,) change counts from `lib.ancestral_char`
    An edge without a change gets half of one; the edited fraction is capped at
    `max_fraction`.  Times are clipped to [T_MIN, T_MAX].
    """
    e = np.asarray(edge, dtype=np.int64).reshape(-1, 2)
    k = np.asarray(changes, dtype=np.float64).reshape(-1)
    if len(k) != len(e):
        raise ValueError("one change count per edge is needed")
    if rate <= 0:
        raise ValueError("rate must be positive")
    par = e[:, 0] - int(ntip)
    if par.size and (par.min() < 0 or par.max() >= node_states.shape[0]):
        raise ValueError("edge parents must be internal nodes covered by node_states")
    n0 = (np.asarray(node_states) == 0).sum(axis=1).astype(np.float64)[par]  # per node, then per edge
    frac = np.minimum(np.maximum(k, 0.5) / np.maximum(n0, 1.0), max_fraction)
    return np.clip(-np.log1p(-frac) / rate, T_MIN, T_MAX)
