"""CPU ORACLE -- TEST INFRASTRUCTURE ONLY.  A plain restatement of the reference's GCMF
text-layer reader, used by tests/ to check the engine's parallel reader
(gcmfgh_read_text_layer).  Reference paths are relative to the reference repository.

  getVertex                           SEQ_Overlay.h:101-118
  CoordToMBR (type 1)                 SEQ_Overlay.h:69-97
  ReadTextFormatPolygon2WithVector    SEQ_Overlay.h:285-390

Deviations shared with the engine and stated there: lines are not cut at MAX_BUFF,
polygons are not limited to MAX_VERTICES, and the MBR extremes start at +/-infinity
instead of +/-1,000,000 (:309-312).
"""
from __future__ import annotations

import re

import numpy as np

_TOK = set("0123456789.-")


def _atof(tok: str) -> float:
    """atof: the longest valid prefix, 0.0 when there is none."""
    for end in range(len(tok), 0, -1):
        try:
            return float(tok[:end])
        except ValueError:
            continue
    return 0.0


def get_vertex(buf: str, i: int, n: int):
    """getVertex: n tokens of [0-9.-] from position i; returns (values, tokens, next i),
    next i == -1 when the buffer was exhausted (SEQ_Overlay.h:116-117)."""
    vals, toks = [], []
    L = len(buf)
    for _ in range(n):
        while i < L and buf[i] not in _TOK:
            i += 1
        j = i
        while i < L and buf[i] in _TOK:
            i += 1
        toks.append(buf[j:i])
        vals.append(_atof(buf[j:i]))
    if i >= L:
        i = -2
    return vals, toks, i + 1


def coord_to_mbr(tok: str) -> int:
    """CoordToMBR(ct, 1): sign and digits with at most 12 fraction digits, padded to 12."""
    out, frac, dot = [], 0, False
    for ch in tok:
        if ch != ".":
            if frac < 12:
                out.append(ch)
                if dot:
                    frac += 1
            else:
                break
        else:
            dot = True
    out.extend("0" * (12 - frac))
    s = "".join(out)
    # atoll: optional sign then digits
    k, sign = 0, 1
    if k < len(s) and s[k] in "+-":
        sign = -1 if s[k] == "-" else 1
        k += 1
    num = 0
    while k < len(s) and s[k].isdigit():
        num = num * 10 + int(s[k])
        k += 1
    return sign * num + 9000000000000000


def read_text_layer(path, with_mbrs=False):
    """Returns (coords (V,2), vnum, ids) of the stored polygons; with_mbrs adds the
    reader's two MBR forms per polygon (SEQ_Overlay.h:327-334): the decimal keys
    CoordToMBR(token) (n,4) uint64 and atof(token) (n,4) float64, both over the header
    pairs and the vertices, in (x1, y1, x2, y2) order."""
    coords, vnum, ids, keys, mbrs = [], [], [], [], []
    with open(path) as f:
        content = f.read()
    lines = re.findall(r"[^\n]*\n|[^\n]+$", content)  # fgets: each line with its newline
    for li, buf in enumerate(lines):
        if li == 0:
            continue                                   # header (:303-306)
        (pid,), _, i = get_vertex(buf, 0, 1)
        pts = []
        x1 = y1 = float("inf")
        x2 = y2 = float("-inf")
        cx1 = cy1 = cx2 = cy2 = None
        while i != -1:
            (a, b), (ta, tb), i = get_vertex(buf, i, 2)
            if i == -1 and a == 0 and b == 0:
                break
            pts.append((a, b))
            if a < x1:
                x1, cx1 = a, ta
            if b < y1:
                y1, cy1 = b, tb
            if a > x2:
                x2, cx2 = a, ta
            if b > y2:
                y2, cy2 = b, tb
        if len(pts) < 2 or cx1 is None:
            continue
        if coord_to_mbr(cx1) == coord_to_mbr(cx2) or coord_to_mbr(cy1) == coord_to_mbr(cy2):
            continue                                   # "MBR Error!" (:331-339)
        if x1 == x2 or y1 == y2:
            continue
        body = pts[2:]
        coords.extend(body)
        vnum.append(len(body))
        ids.append(int(pid))
        keys.append([coord_to_mbr(t) for t in (cx1, cy1, cx2, cy2)])
        mbrs.append([_atof(t) for t in (cx1, cy1, cx2, cy2)])
    out = (np.array(coords, np.float64).reshape(-1, 2), np.array(vnum, np.int32), np.array(ids, np.int64))
    if with_mbrs:
        out += (np.array(keys, np.uint64).reshape(-1, 4), np.array(mbrs, np.float64).reshape(-1, 4))
    return out
