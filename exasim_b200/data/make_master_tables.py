"""Extract the reference-element node sets and quadrature rules used by Exasim's
preprocessor into a compact table shipped with this package.

Exasim's preprocessor looks both up in two binary tables
(text2code/text2code/masternodes.bin and gaussnodes.bin, read by
``masternodes()`` / ``gaussnodes()`` in text2code/text2code/makemaster.cpp:83-231).
Both are numeric data (node coordinates, face-node permutations, quadrature
points and weights), indexed column-major by (field, elemtype, order, dim).
This script copies the entries for element types 0 (simplex) and 1 (tensor),
dimensions 1-3, polynomial orders 1-6 and quadrature orders 1-12 into
``master_tables.npz`` so that synthetic inputs can be generated where the
reference tree is absent.

Usage:  python make_master_tables.py <path to text2code/text2code>
"""
import os
import sys

import numpy as np


def _load(fn):
    t = np.fromfile(fn, dtype=np.float64)
    nd = int(t[0])
    na = t[1:1 + nd].astype(np.int64)
    off = 1 + nd
    tb = int(np.prod(na))
    s1 = t[off:off + tb].astype(np.int64)
    s2 = t[off + tb:off + 2 * tb].astype(np.int64)
    lz = np.concatenate([[0], np.cumsum(s1 * s2)])
    return t, na, s1, s2, lz, off + 2 * tb


def _block(tab, i, e, p, d):
    t, na, s1, s2, lz, ds = tab
    idx = i + na[0] * (e + na[1] * ((p - 1) + na[2] * (d - 1)))
    return t[ds + lz[idx]: ds + lz[idx + 1]].copy(), (int(s1[idx]), int(s2[idx]))


def main(src):
    nodes = _load(os.path.join(src, "masternodes.bin"))
    gauss = _load(os.path.join(src, "gaussnodes.bin"))
    out = {}
    for e in (0, 1):
        for d in (1, 2, 3):
            for p in range(1, 7):
                if p > nodes[1][2]:
                    continue
                for i, name in enumerate(("xpe", "telem", "xpf", "tface", "perm")):
                    v, shp = _block(nodes, i, e, p, d)
                    out[f"n_{e}_{d}_{p}_{name}"] = v
                    out[f"n_{e}_{d}_{p}_{name}_shape"] = np.array(shp)
            for q in range(1, 13):
                if q > gauss[1][2]:
                    continue
                for i, name in enumerate(("x", "w")):
                    v, shp = _block(gauss, i, e, q, d)
                    out[f"g_{e}_{d}_{q}_{name}"] = v
                    out[f"g_{e}_{d}_{q}_{name}_shape"] = np.array(shp)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "master_tables.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, os.path.getsize(dst), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.environ["EXASIM_REF"], "text2code/text2code"))
