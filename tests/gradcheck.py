"""Element-wise gradient parity bar shared by the GPU gradient tests.

For every entry i of a gradient table:

    |g_i - g_ref_i| <= REL * |g_ref_i| + (KAPPA + n_i) * 2^-24 * mass_i

g_ref is the FP64 oracle's gradient.  mass_i is the oracle's FP32 error
budget of that entry (``forward_backward(..., want_mass=True)``): the sum,
over the contributions that form entry i, of the magnitudes an FP32
evaluation of the same contract rounds — the transmittance product, each
1 - alpha (one rounding of 1), the SH sum, dL/dC through the ray colour, the
suffix C - P_k — propagated to first order; KAPPA covers that budget's
dropped constants.  n_i is the entry's number of terms: the device adds them
up with float atomics in no fixed order, and any order of n FP32 additions
errs by at most (n - 1) 2^-24 times the sum of the terms' magnitudes, which
the mass bounds.  REL = 1e-4 is the relative bar for FP32 arithmetic.  The
second term is what FP32 cannot resolve: an entry whose contributions cancel,
or one reached only behind a near-opaque cell, is held to the error its own
terms allow, and an entry with no contributions (mass 0) must be exactly 0.

Set BV_PARITY_LOG to a file path to append one JSON line per checked table:
the largest fraction of the bound used and the median relative error.
"""

from __future__ import annotations

import json
import os

import numpy as np

REL = 1e-4
KAPPA = 16.0
U = 2.0 ** -24


def check(name, got, ref, mass, count, rel=REL, kappa=KAPPA, where=""):
    got = np.asarray(got, np.float64).reshape(-1)
    ref = np.asarray(ref, np.float64).reshape(-1)
    mass = np.asarray(mass, np.float64).reshape(-1)
    count = np.asarray(count, np.float64).reshape(-1)
    assert got.shape == ref.shape == mass.shape == count.shape, (name, got.shape, ref.shape)
    assert np.isfinite(got).all(), name
    err = np.abs(got - ref)
    bound = rel * np.abs(ref) + (kappa + count) * U * mass
    with np.errstate(divide="ignore", invalid="ignore"):
        used = np.where(bound > 0, err / bound, np.where(err > 0, np.inf, 0.0))
        relerr = np.where(np.abs(ref) > 0, err / np.abs(ref), 0.0)
    nz = np.abs(ref) > 0
    stats = {"table": name, "where": where, "entries": int(got.size), "nonzero": int(nz.sum()),
             "max_bound_used": float(used.max()) if used.size else 0.0,
             "max_terms": int(count.max()) if count.size else 0,
             "median_rel_err": float(np.median(relerr[nz])) if nz.any() else 0.0,
             "p99_rel_err": float(np.quantile(relerr[nz], 0.99)) if nz.any() else 0.0,
             "norm_rel_err": float(np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300))}
    log = os.environ.get("BV_PARITY_LOG")
    if log:
        with open(log, "a") as f:
            f.write(json.dumps(stats) + "\n")
    bad = np.flatnonzero(used > 1.0)
    assert bad.size == 0, (name, where, f"{bad.size} entries over the bound", stats,
                           [(int(i), got[i], ref[i], mass[i], count[i]) for i in bad[:5]])
    return stats


def check_all(got: dict, ref: dict, where="", tables=("density", "sh", "pos", "radius"), **kw):
    """Checks every gradient table present in both the device output (keys
    d_<table>) and the oracle output (d_<table>, mass_<table>,
    count_<table>); every table is checked before a failure is raised."""
    out, failures = [], []
    for t in tables:
        g, r, m = got.get("d_" + t), ref.get("d_" + t), ref.get("mass_" + t)
        if g is None or r is None or m is None:
            continue
        try:
            out.append(check(t, g, r, m, ref["count_" + t], where=where, **kw))
        except AssertionError as e:
            failures.append(e)
    if failures:
        raise failures[0]
    return out
