"""Vioreanu-Rokhlin table access for host-side input preparation (the same
numbers as csrc/vr_table.h, parsed once)."""
import os
import re

import numpy as np

_cache = None


def _load():
    global _cache
    if _cache is None:
        t = open(os.path.join(os.path.dirname(__file__), "csrc", "vr_table.h")).read()
        off = [int(x) for x in re.search(r"offset\[22\] = \{\s*([^}]*)\}", t).group(1).split(",")]
        uv = np.array([float(x) for x in re.search(r"qol_vr_uv\[\d+\] = \{(.*?)\};", t, re.S).group(1).split(",") if x.strip()])
        w = np.array([float(x) for x in re.search(r"qol_vr_w\[\d+\] = \{(.*?)\};", t, re.S).group(1).split(",") if x.strip()])
        _cache = (off, uv, w)
    return _cache


def nodes(deg):
    off, uv, w = _load()
    a, b = off[deg], off[deg + 1]
    return uv[2 * a:2 * b].reshape(-1, 2).copy(), w[a:b].copy()
