"""The chunked first-fit that the grouping kernels run, as a plain-Python model.

A group only ever gains members (qwc: its basis gains bits), so the groups that
accept a term only become fewer as terms are placed.  The device code relies on
that: the first group accepting a term at the start of its chunk is a lower
bound on the group it joins, and in full mode the groups that accepted it then
need checking only against members added during the chunk.  This model follows
those steps (bound pass, window mask, fast check of the bound, ordered slow
path) and must reproduce the sequential first-fit for every chunk length.
"""

from __future__ import annotations

import numpy as np
import pytest


def _terms(rng, n_terms, words, p):
    x = (rng.random((n_terms, words, 64)) < p)
    z = (rng.random((n_terms, words, 64)) < p)
    pack = lambda b: [int("".join("1" if v else "0" for v in row[::-1]), 2) for row in b.reshape(n_terms, -1)]
    return list(zip(pack(x), pack(z)))


def _qwc_ok(t, basis):
    return ((t[0] & basis[1]) ^ (t[1] & basis[0])) == 0


def _commute(a, b):
    return bin((a[0] & b[1]) ^ (a[1] & b[0])).count("1") % 2 == 0


def first_fit(terms, full):
    groups, basis, out = [], [], []
    for t in terms:
        for g in range(len(groups)):
            if (all(_commute(t, terms[m]) for m in groups[g]) if full else _qwc_ok(t, basis[g])):
                break
        else:
            g = len(groups)
            groups.append([])
            basis.append((0, 0))
        groups[g].append(len(out))
        basis[g] = (basis[g][0] | t[0], basis[g][1] | t[1])
        out.append(g)
    return out


def chunked_first_fit(terms, full, chunk, window=32):
    groups, basis, out = [], [], []
    accepts = lambda t, g: all(_commute(t, terms[m]) for m in groups[g]) if full else _qwc_ok(t, basis[g])
    for c0 in range(0, len(terms), chunk):
        c1 = min(len(terms), c0 + chunk)
        g0 = len(groups)
        # bound pass: first accepting group at the chunk's start, and the window mask
        bounds, masks = [], []
        for t in terms[c0:c1]:
            lb = next((g for g in range(g0) if accepts(t, g)), g0)
            bounds.append(lb)
            masks.append([lb + j < g0 and accepts(t, lb + j) for j in range(window)])
        for k, t in enumerate(terms[c0:c1]):
            lb = bounds[k]
            chunk_members = lambda g: [m for m in groups[g] if m >= c0] if g < g0 else groups[g]
            chunk_ok = lambda g: all(_commute(t, terms[m]) for m in chunk_members(g))
            best = None
            if full:
                if lb < g0 and chunk_ok(lb):
                    best = lb
                else:
                    cands = [lb + j for j in range(1, window) if lb < g0 and masks[k][j]]
                    best = next((g for g in cands if chunk_ok(g)), None)
                    if best is None:
                        best = next((g for g in range(lb + window, g0) if accepts(t, g)), None)
                    if best is None:
                        best = next((g for g in range(g0, len(groups)) if chunk_ok(g)), None)
            else:
                best = next((g for g in range(lb, len(groups)) if accepts(t, g)), None)
            if best is None:
                best = len(groups)
                groups.append([])
                basis.append((0, 0))
            groups[best].append(c0 + k)
            basis[best] = (basis[best][0] | t[0], basis[best][1] | t[1])
            out.append(best)
    return out


@pytest.mark.parametrize("full", [False, True])
@pytest.mark.parametrize("n_terms,words,p", [(300, 1, 0.08), (250, 2, 0.03), (200, 1, 0.2)])
def test_chunked_first_fit_equals_first_fit(full, n_terms, words, p):
    rng = np.random.default_rng(20261204 + n_terms + 7 * words + int(full))
    terms = _terms(rng, n_terms, words, p)
    want = first_fit(terms, full)
    for chunk in (1, 3, 17, 64, 1000):
        assert chunked_first_fit(terms, full, chunk) == want, chunk
