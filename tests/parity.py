"""Comparison helpers shared by the parity tests."""
from __future__ import annotations

import numpy as np
import torch

REL_TOL = 2e-6  # stated tolerance for distances and hit points across traversal orders


def to_np(rec) -> dict:
    out = {}
    for k, v in vars(rec).items():
        out[k] = v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else v
    return out


def assert_bitwise(gpu: dict, ref: dict, fields, what=""):
    for f in fields:
        a, b = np.asarray(gpu[f]), np.asarray(ref[f])
        assert a.shape == b.shape, f"{what}{f}: shape {a.shape} vs {b.shape}"
        if a.dtype == np.bool_ or b.dtype == np.bool_:
            bad = a.astype(bool) != b.astype(bool)
        elif a.dtype.kind == "f":
            # bit for bit, except that NaN in both counts as equal: the payload of a NaN
            # (degenerate triangle normals) differs between the GPU and x86
            a32, b32 = a.astype(np.float32), b.astype(np.float32)
            bad = (a32.view(np.uint32) != b32.view(np.uint32)) & ~(np.isnan(a32) & np.isnan(b32))
        else:
            bad = a.astype(np.int64) != b.astype(np.int64)
        nbad = int(np.count_nonzero(bad))
        if nbad:
            idx = np.argwhere(bad)[:5]
            raise AssertionError(f"{what}{f}: {nbad} mismatches, first at {idx.tolist()}: "
                                 f"gpu={a[tuple(idx[0])]!r} ref={b[tuple(idx[0])]!r}")


def tie_report(a: dict, b: dict, rel=REL_TOL) -> dict:
    """Compares two result sets that may differ only at ties: same validity; where the
    primitive differs, the distances agree within `rel` (relative)."""
    va, vb = np.asarray(a["valid"]).astype(bool), np.asarray(b["valid"]).astype(bool)
    pa, pb = np.asarray(a["prim_id"]), np.asarray(b["prim_id"])
    da, db = np.asarray(a["d"], np.float64), np.asarray(b["d"], np.float64)
    both = va & vb
    scale = np.maximum(np.maximum(np.abs(da), np.abs(db)), 1e-30)
    reldiff = np.abs(da - db) / scale
    prim_diff = both & (pa != pb)
    return {
        "n": int(va.size),
        "valid_mismatch": int(np.count_nonzero(va != vb)),
        "prim_mismatch": int(np.count_nonzero(prim_diff)),
        "prim_mismatch_exact_tie": int(np.count_nonzero(prim_diff & (da == db))),
        "prim_mismatch_not_tie": int(np.count_nonzero(prim_diff & (reldiff > rel))),
        "max_rel_d": float(reldiff[both].max()) if both.any() else 0.0,
    }


def sil_variant_report(exact: dict, variant: dict, brute: dict, rel=REL_TOL) -> dict:
    """Like tie_report for a fast silhouette variant against the exact one, with one more
    allowance: the reference's normal-cone test may reject a node that holds the true
    nearest silhouette (its cones reuse face 0's normal and measure their radius from edge
    midpoints), while the fast variants' cone test admits every node the reference admits
    and sometimes more.  A variant answer that is strictly nearer than the exact one and
    equals the brute-force nearest silhouette is counted in `nearer_true`, not as a
    mismatch; every other differing primitive must be a tie."""
    va, vv = np.asarray(exact["valid"]).astype(bool), np.asarray(variant["valid"]).astype(bool)
    de, dv = np.asarray(exact["d"], np.float64), np.asarray(variant["d"], np.float64)
    db = np.asarray(brute["d"], np.float64)
    vb = np.asarray(brute["valid"]).astype(bool)
    scale = np.maximum(np.maximum(np.abs(de), np.abs(dv)), 1e-30)
    nearer_true = va & vv & vb & (dv < de) & (np.abs(dv - db) <= rel * np.maximum(np.abs(db), 1e-30))
    keep = ~nearer_true
    rep = tie_report({k: np.asarray(exact[k])[keep] for k in ("valid", "prim_id", "d")},
                     {k: np.asarray(variant[k])[keep] for k in ("valid", "prim_id", "d")}, rel)
    rep["nearer_true"] = int(np.count_nonzero(nearer_true))
    rep["max_rel_gain"] = float(((de - dv) / scale)[nearer_true].max()) if nearer_true.any() else 0.0
    return rep


def assert_sil_variant(exact: dict, variant: dict, brute: dict, what="", max_nearer=0.01):
    rep = sil_variant_report(exact, variant, brute)
    ok = (rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL
          and rep["nearer_true"] <= max_nearer * rep["n"])
    assert ok, (what, rep)
