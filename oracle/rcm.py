"""Independent restatement of the library's reverse Cuthill-McKee ordering
(mgpu_rcm_order). TEST INFRASTRUCTURE: the bit-exact check of the library's
integer result, and the cell order the CPU reference leg of bench.py builds
its input mesh with.

Start of each component: the unvisited cell of least (degree, index), moved to
a pseudo-peripheral cell (George-Liu: BFS, restart from the least (degree,
index) cell of the last level while the eccentricity grows). Neighbours are
queued in (degree, index) order; the visit order is reversed.
"""
from collections import deque

import numpy as np


def adjacency(mesh):
    n = mesh.ncells
    i = mesh.c1 > 0
    a = mesh.c0[i].astype(np.int64) - 1
    b = mesh.c1[i].astype(np.int64) - 1
    src = np.concatenate([a, b])
    dst = np.concatenate([b, a])
    key = np.unique(src * n + dst)
    src, dst = key // n, key % n
    ptr = np.searchsorted(src, np.arange(n + 1))
    dst = dst.tolist()
    return [dst[ptr[k]:ptr[k + 1]] for k in range(n)]


def rcm(mesh) -> np.ndarray:
    adj = adjacency(mesh)
    n = len(adj)
    deg = [len(a) for a in adj]
    key = lambda v: (deg[v], v)
    visited = [False] * n

    def bfs_last(r):
        seen = {r}
        cur = [r]
        ecc = 0
        while True:
            nxt = []
            for v in cur:
                for w in adj[v]:
                    if not visited[w] and w not in seen:
                        seen.add(w)
                        nxt.append(w)
            if not nxt:
                return ecc, cur
            ecc += 1
            cur = nxt

    order = []
    cand = sorted(range(n), key=key)
    ci = 0
    while len(order) < n:
        while visited[cand[ci]]:
            ci += 1
        r = cand[ci]
        ecc, last = bfs_last(r)
        while True:
            x = min(last, key=key)
            ex, lx = bfs_last(x)
            if ex > ecc:
                r, ecc, last = x, ex, lx
            else:
                break
        q = deque([r])
        visited[r] = True
        while q:
            v = q.popleft()
            order.append(v)
            for w in sorted((w for w in adj[v] if not visited[w]), key=key):
                visited[w] = True
                q.append(w)
    new_of_old = np.zeros(n, np.int32)
    for p in range(n):
        new_of_old[order[n - 1 - p]] = p + 1
    return new_of_old
