"""Comparison of one oracle kernel with the reference's kernel on the same state.

Two reference kernels race on purpose-free data (their results depend on
thread timing), so for them a per-cell result is accepted when it equals the
oracle's result under either interleaving:

* d_FreeSurface2D_1 (lbmKernel2D.cu:36 vs :116): a cell's outgoing load and a
  neighbour's reconstruction store to the same slot.  "pre": the load sees the
  old population (the oracle's default); "post": it sees the rebuilt one
  (OracleConfig.fs1_post).
* d_FreeSurface2D_4 (lbmKernel2D.cu:290-294 vs :249-267): a cell counts a
  neighbour's flag while the neighbour converts it.  "post": converted flags
  (default); "pre": unconverted (OracleConfig.fs_count_pre).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from oracle import oracle as O

FIELDS_FS = ("f", "rho", "u", "flags", "mass", "excess", "phi")


def snapshot(o, fs=True) -> dict:
    keys = FIELDS_FS if fs else ("f", "rho", "u", "flags")
    return {k: getattr(o, k).copy() for k in keys}


def oracle_with_state(geo, cfg: O.OracleConfig, state: dict, t: int, **overrides) -> O.Oracle:
    o = O.Oracle(geo, dataclasses.replace(cfg, **overrides))
    for k, v in state.items():
        getattr(o, k)[:] = v
    o.t = t
    return o


def either(ref, a, b) -> np.ndarray:
    """Per-element: ref equals a or b (value equality, NaN equal)."""
    def eq(x, y):
        return (x == y) | (np.isnan(x) & np.isnan(y)) if np.asarray(x).dtype.kind == "f" else (x == y)
    return eq(ref, a) | eq(ref, b)


def check_kernel(geo, cfg: O.OracleConfig, state: dict, t: int, kid: int, ref: dict, what: str = "") -> dict:
    """Runs oracle kernel kid on state and checks it against the reference's
    output fields ``ref`` (a dict of full arrays; key ``f`` may instead be
    given as sparse ``f_idx``/``f_val``).  Returns the oracle's (default
    interleaving) output state and the number of cells decided by the race."""
    o = oracle_with_state(geo, cfg, state, t)
    o.kernel(kid)
    out = snapshot(o, cfg.free_surface)
    alt = None
    if kid == O.K_FS1:
        a = oracle_with_state(geo, cfg, state, t, fs1_post=True)
        a.kernel(kid)
        alt = snapshot(a, cfg.free_surface)
    elif kid == O.K_FS4:
        a = oracle_with_state(geo, cfg, state, t, fs_count_pre=True)
        a.kernel(kid)
        alt = snapshot(a, cfg.free_surface)
    raced = 0
    for k, r in ref.items():
        if k == "f_idx":
            continue
        if k == "f_val":
            idx = ref["f_idx"]
            mine_full = out["f"]
            # every slot the reference changed must match, and no other slot may change in the oracle
            cand = mine_full[idx]
            ok = either(r, cand, alt["f"][idx]) if alt is not None else (r == cand)
            assert ok.all(), f"{what} f: reference-changed slots differ"
            changed_o = np.nonzero(mine_full != state["f"])[0]
            extra = np.setdiff1d(changed_o, idx)
            if alt is not None:
                extra = extra[alt["f"][extra] == state["f"][extra]] if extra.size else extra
            assert extra.size == 0, f"{what} f: oracle changed slots the reference kept ({extra[:5]})"
            continue
        mine = out[k]
        if alt is None or k in ("flags",):
            bad = ~either(r, mine, mine)
            assert not bad.any(), f"{what} {k}: first mismatch at {np.nonzero(bad)[0][:5]}"
        else:
            ok = either(r, mine, alt[k])
            assert ok.all(), f"{what} {k}: mismatch at {np.nonzero(~ok)[0][:5]}"
            raced += int((~either(r, mine, mine)).sum())
    return dict(state=out, raced=raced)
