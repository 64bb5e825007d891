"""Minimal reader for Fluent ASCII .cas meshes (sections 10, 12, 13, 45).

Used only by make_golden.py (fixture generation in a checkout where the
reference's case files exist). Follows the record layout handled by the
reference's reader, src/unstructured/mod_uns_cas_reader.f90:44-523: integers
are hexadecimal, a face record lists its nodes then c0 c1, and ftype 0 means
each face carries its own node count.
"""
from __future__ import annotations

import re

import numpy as np

from mixsolver_b200.meshgen import FaceMesh

_TOK = re.compile(r'"[^"]*"|\(|\)|[^\s()]+')


def read_cas(path: str) -> FaceMesh:
    text = open(path, "r", errors="replace").read()
    toks = _TOK.findall(text)
    pos = 0
    n = len(toks)
    nodes = {}
    faces = []          # (first, nodes-list-array, c0, c1, zone)
    ncells = 0
    zone_names = {}

    def skip_group(p):
        depth = 0
        while p < n:
            t = toks[p]
            if t == "(":
                depth += 1
            elif t == ")":
                depth -= 1
                if depth == 0:
                    return p + 1
            p += 1
        return p

    while pos < n:
        if toks[pos] != "(":
            pos += 1
            continue
        sec = toks[pos + 1] if pos + 1 < n else ""
        if sec not in ("10", "12", "13", "45"):
            pos = skip_group(pos)
            continue
        # header group
        p = pos + 2
        if toks[p] != "(":
            pos = skip_group(pos)
            continue
        q = p + 1
        hdr = []
        while toks[q] != ")":
            hdr.append(toks[q]); q += 1
        q += 1
        if sec == "45":
            zid = int(hdr[0])
            zone_names[zid] = hdr[1] if len(hdr) > 1 else ""
            pos = skip_group(pos)
            continue
        try:
            h = [int(v, 16) for v in hdr[:5]]
        except ValueError:
            pos = skip_group(pos)
            continue
        if toks[q] != "(":           # declaration record without payload
            if sec == "12" and h[0] == 0:
                ncells = max(ncells, h[2])
            pos = skip_group(pos)
            continue
        # payload group
        r = q + 1
        body = []
        while toks[r] != ")":
            body.append(toks[r]); r += 1
        if sec == "10":
            zid, first, last = h[0], h[1], h[2]
            nd = h[4] if len(h) > 4 else 3
            vals = np.array([float(v) for v in body]).reshape(-1, nd)
            for k in range(last - first + 1):
                xyz = np.zeros(3)
                xyz[:nd] = vals[k]
                nodes[first + k] = xyz
        elif sec == "12":
            ncells = max(ncells, h[2])
        elif sec == "13":
            zid, first, last, ftype = h[0], h[1], h[2], h[4]
            ints = [int(v, 16) for v in body]
            pp = 0
            for k in range(last - first + 1):
                if ftype == 0:
                    ft = ints[pp]; pp += 1
                else:
                    ft = ftype
                if ft == 5:
                    nn = ints[pp]; pp += 1
                else:
                    nn = ft
                fn = ints[pp:pp + nn]; pp += nn
                c0, c1 = ints[pp], ints[pp + 1]; pp += 2
                faces.append((first + k, fn, c0, c1, zid))
        pos = skip_group(pos)

    nn = max(nodes) if nodes else 0
    x = np.zeros((nn, 3))
    for k, v in nodes.items():
        x[k - 1] = v
    faces.sort(key=lambda t: t[0])
    cnt = np.array([len(f[1]) for f in faces], np.int64)
    ptr = np.zeros(len(faces) + 1, np.int64)
    np.cumsum(cnt, out=ptr[1:])
    fnodes = np.concatenate([np.asarray(f[1], np.int32) for f in faces])
    c0 = np.array([f[2] for f in faces], np.int32)
    c1 = np.array([f[3] for f in faces], np.int32)
    zone = np.array([f[4] for f in faces], np.int32)
    return FaceMesh(x, ptr.astype(np.int32), fnodes, c0, c1, zone, int(ncells), zone_names)
