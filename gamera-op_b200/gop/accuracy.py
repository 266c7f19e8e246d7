"""Error measures of a result against a reference result.

``rel_l1`` is the relative L1 error of each variable over the active cells
(and every evolved face of the face fields).  Scalars (rho, p) are
normalised by their own L1 norm; vector components by the L1 norm of the
vector's magnitude, so a component that is zero up to round-off in the
reference (e.g. v_y of a field loop advected along x) is judged against the
size of the vector it belongs to rather than against its own noise.
"""
from __future__ import annotations

import numpy as np

NG = 4


def _views(n, res):
    sl = tuple(slice(NG, NG + m) for m in n)
    gas = [res["gas"][m][sl] for m in range(5)]
    faces = []
    for a in range(3):
        s = list(sl)
        s[a] = slice(NG, NG + n[a] + 1)
        faces.append(res["face_b"][a][tuple(s)])
    return gas, faces


def rel_l1(n, got, want) -> dict:
    """Per-variable relative L1 (rho v1 v2 v3 p B1 B2 B3) of ``got``
    against ``want``; both hold "gas" and "face_b" in the reference layout."""
    g, gf = _views(n, got)
    w, wf = _views(n, want)
    out = {}
    for m, name in ((0, "rho"), (4, "p")):
        den = np.abs(w[m]).sum()
        out[name] = float(np.abs(g[m] - w[m]).sum() / den) if den > 0 else float(np.abs(g[m] - w[m]).sum())
    speed = np.sqrt(w[1] ** 2 + w[2] ** 2 + w[3] ** 2).sum()
    for a in range(3):
        num = np.abs(g[1 + a] - w[1 + a]).sum()
        out[f"v{a + 1}"] = float(num / speed) if speed > 0 else float(num)
    # |B| from the faces' mean magnitude per axis (face arrays differ in shape)
    bmag = sum(np.abs(wf[a]).mean() for a in range(3))
    for a in range(3):
        num = np.abs(gf[a] - wf[a]).mean()
        out[f"B{a + 1}"] = float(num / bmag) if bmag > 0 else float(num)
    return out


def worst(errs: dict):
    """(largest error, its variable)."""
    k = max(errs, key=errs.get)
    return errs[k], k
