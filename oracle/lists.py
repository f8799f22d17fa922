"""CPU restatement of this library's FMM interaction-list rule (test infrastructure).

The reference builds per-box lists on an adaptive median-split tree
(``src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmmsort.cpp:792-910``) with two checks per
box pair (``fmm.cpp:1735-1835``): the theta criterion r1 + r2 <= theta d and,
with THETACUTOFFCHECK, the cutoff check d - r1 - r2 >= cutoff.  The library
uses a uniform quadtree, where these checks depend only on the integer box
offset, so it builds offset tables instead; this module restates that
construction independently, in plain Python, so the tables the library builds
can be compared bit for bit, and checks that every (target leaf, source leaf)
pair is covered exactly once (by P2P or by one M2L at one level).
"""
import math


def well_separated(i, j, w, cutoff, theta):
    s2 = float(i * i + j * j)
    return (s2 * (theta * theta) >= 2.0) and ((math.sqrt(s2) - math.sqrt(2.0)) * w >= cutoff)


def _fd2(a):
    return a // 2  # Python floor division == floor for negatives


def build(L, kb, w0, cutoff, theta=0.5):
    """Return dict(near=[set per level], far=[None, [list per pos] per level],
    p2p=sorted list, nleaf=[set per block position])."""
    near = []
    for l in range(L + 1):
        ext = (1 << l) - 1
        w = math.ldexp(w0, -l)
        rmax = max(math.sqrt(2.0) / theta, cutoff / w + math.sqrt(2.0))
        R = int(min(ext, math.ceil(rmax) + 1.0))
        near.append({(i, j) for i in range(-R, R + 1) for j in range(-R, R + 1)
                     if not well_separated(i, j, w, cutoff, theta)})
    B = 1 << kb
    extL = (1 << L) - 1
    q = {(o[0] + cx, o[1] + cy) for cx in range(B) for cy in range(B) for o in near[L]}
    nleaf = [None] * (B * B)
    for cx in range(B):
        for cy in range(B):
            nleaf[cx + B * cy] = {(a - cx, b - cy) for (a, b) in q
                                  if abs(a - cx) <= extL and abs(b - cy) <= extL}
    if L >= 1:
        ext = (1 << (L - 1)) - 1
        for cx in range(B):
            for cy in range(B):
                c0, c1 = cx & 1, cy & 1
                for (oi, oj) in nleaf[cx + B * cy]:
                    p = (_fd2(c0 + oi), _fd2(c1 + oj))
                    if abs(p[0]) <= ext and abs(p[1]) <= ext:
                        near[L - 1].add(p)
        for l in range(L - 1, 0, -1):
            ext = (1 << (l - 1)) - 1
            for c0 in (0, 1):
                for c1 in (0, 1):
                    for (oi, oj) in list(near[l]):
                        p = (_fd2(c0 + oi), _fd2(c1 + oj))
                        if abs(p[0]) <= ext and abs(p[1]) <= ext:
                            near[l - 1].add(p)
    far = [None]
    Bp = max(B, 2)
    for l in range(1, L + 1):
        ext = (1 << l) - 1
        npos = Bp * Bp if l == L else 4
        fl = []
        for pos in range(npos):
            if l == L:
                px, py = pos % Bp, pos // Bp
                c0, c1 = px & 1, py & 1
                own = nleaf[(px % B) + B * (py % B)]
            else:
                c0, c1 = pos & 1, (pos >> 1) & 1
                own = near[l]
            f = set()
            for (Oi, Oj) in near[l - 1]:
                for d0 in (0, 1):
                    for d1 in (0, 1):
                        o = (2 * Oi + d0 - c0, 2 * Oj + d1 - c1)
                        if abs(o[0]) > ext or abs(o[1]) > ext or o in own:
                            continue
                        f.add(o)
            fl.append(sorted(f))
        far.append(fl)
    return {"near": [sorted(s) for s in near], "far": far, "p2p": sorted(q), "nleaf": nleaf,
            "L": L, "kb": kb}


def flatten(t):
    out = [t["L"], t["kb"]]
    for l in range(t["L"] + 1):
        out.append(len(t["near"][l]))
        for o in t["near"][l]:
            out += [o[0], o[1]]
    for l in range(1, t["L"] + 1):
        out.append(len(t["far"][l]))
        for f in t["far"][l]:
            out.append(len(f))
            for o in f:
                out += [o[0], o[1]]
    out.append(len(t["p2p"]))
    for o in t["p2p"]:
        out += [o[0], o[1]]
    return out


def coverage_counts(t):
    """For every (target leaf T, source leaf S) of the 2^L grid, how many times
    the pair is handled: 1 if S is in T's P2P set, plus 1 for every level l at
    which S's ancestor is in the M2L list of T's ancestor.  Returns the set of
    distinct counts (must be {1})."""
    L, kb = t["L"], t["kb"]
    B = 1 << kb
    Bp = max(B, 2)
    G = 1 << L
    farsets = [None] + [[set(f) for f in t["far"][l]] for l in range(1, L + 1)]
    counts = set()
    for tx in range(G):
        for ty in range(G):
            cb = (tx % B) + B * (ty % B)
            near = t["nleaf"][cb]
            for sx in range(G):
                for sy in range(G):
                    c = 1 if (sx - tx, sy - ty) in near else 0
                    for l in range(1, L + 1):
                        sh = L - l
                        ax, ay, bx, by = tx >> sh, ty >> sh, sx >> sh, sy >> sh
                        pos = (ax % Bp) + Bp * (ay % Bp) if l == L else (ax & 1) | ((ay & 1) << 1)
                        if (bx - ax, by - ay) in farsets[l][pos]:
                            c += 1
                    counts.add(c)
    return counts


def leaf_keys(x, y, x0, y0, w, L):
    """Leaf Morton keys: qx = clamp(floor((x - x0)/w), 0, 2^L - 1), x bits even."""
    import numpy as np
    hi = (1 << L) - 1
    qx = np.clip(np.floor((np.asarray(x) - x0) / w), 0, hi).astype(np.uint64)
    qy = np.clip(np.floor((np.asarray(y) - y0) / w), 0, hi).astype(np.uint64)
    key = np.zeros_like(qx)
    for b in range(L):
        key |= ((qx >> np.uint64(b)) & np.uint64(1)) << np.uint64(2 * b)
        key |= ((qy >> np.uint64(b)) & np.uint64(1)) << np.uint64(2 * b + 1)
    return key.astype(np.uint32)
