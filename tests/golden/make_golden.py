"""Generates the golden fixtures under tests/golden/ (committed; this script is
re-run only when a fixture changes).

clustering_kn{0..4}.npz
    Digis of the reference's clustering known-answer test (test/gpu_clustering_t.jl,
    generateClusters(kn) at lines 27-215) with the expected cluster count `ncl` that the
    test asserts equals sum(nClustersInModule) (line 278). The digi pattern is restated
    here from the test's description: big noise, edge columns, diagonals, messy and
    holed clusters, invalid digis, and modules 11..1799.
clustering_diag8.npz
    plugin-SiPixelClusterizer/testClustering.jl:13-35: 8 pixels on a diagonal, 6 clusters.
brokenline_fixtures.json
    The 3-, 4- and 5-hit fixtures of test/testBrokenLine.jl:12-72 with B = 0.0113921
    (line 81), read from that file, plus the CPU oracle's FP64 fit of each. The reference
    test prints and asserts nothing, so the fit values are oracle-generated goldens.

Usage: python tests/golden/make_golden.py --reference <root of a CMS-Julia checkout>
"""
from __future__ import annotations

import argparse
import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
INV_ID = 9999


def generate_clusters(kn: int):
    ids, xs, ys, adcs = [], [], [], []
    ncl = 0

    def push(i, x, y, a):
        ids.append(i); xs.append(x); ys.append(y); adcs.append(a)

    ystep = [5, 7, 9, 1, 3, 0, 4, 8, 2, 6]
    if kn % 2 == 1:  # big noise: isolated pixels of module 666, each its own cluster
        max_pixels = 1000
        done = False
        for x in range(0, 140, 3):
            for yy in range(0, 400, 3):
                ncl += 1
                push(666, x, yy, 1000)
                if max_pixels <= ncl:
                    done = True
                    break
            if done:
                break
    # module 42
    ncl += 1; push(42, 10, 10, 100 if kn == 0 else 5000)          # isolated
    ncl += 1; push(42, 10, 0, 5000)                               # first column
    ncl += 1; push(42, 90, 2, 5000); push(42, 90, 1, 5000)        # first columns, adjacent
    ncl += 1; push(42, 10, 415, 5000)                             # last column
    ncl += 1; push(42, 90, 415, 2500); push(42, 90, 414, 2500)    # last columns, adjacent
    ncl += 1
    for x in range(20, 25):                                      # diagonal
        push(42, x, x, 1000)
    ncl += 1
    for x in range(45, 40, -1):                                  # reversed diagonal
        push(42, x, x, 1000)
    ncl += 1
    push(INV_ID, 0, 0, 0)                                        # an invalid digi
    xx = [21, 25, 23, 24, 22]
    for k in range(5):                                           # messy
        push(42, xx[k], 20 + xx[k], 1000)
    ncl += 1
    for k in range(5):                                           # holes
        push(42, xx[k], 100, 100 if kn == 2 else 1000)
        if xx[k] % 2 == 0:
            push(42, xx[k], 101, 1000)
    ncl += 1; push(0, 10, 10, 5000)                              # module 0
    for mid in range(11, 1800, 2):
        if (mid // 20) % 2 != 0:
            push(INV_ID, 0, 0, 0)
        for x in range(0, 37, 4):
            ncl += 1
            if (mid // 10) % 2 != 0:
                for k in range(10):
                    push(mid, x, x + ystep[k], 100)
                    push(mid, x + 1, x + ystep[k] + 2, 1000)
            else:
                for k in range(9, -1, -1):
                    push(mid, x, x + ystep[k], 10 if kn == 2 else 1000)
                    if ystep[k] == 3:
                        continue  # hole
                    if mid == 51:
                        push(INV_ID, 0, 0, 0); push(INV_ID, 0, 0, 0)
                    push(mid, x + 1, x + ystep[k] + 2, 10 if kn == 2 else 1000)
    return (np.array(ids, np.uint16), np.array(xs, np.int16), np.array(ys, np.int16), np.array(adcs, np.int32), ncl)


def parse_brokenline(ref: Path):
    src = (ref / "src/julia-serial/test/testBrokenLine.jl").read_text()
    vec = lambda s: [float(v) for v in re.findall(r"[-+]?\d*\.\d+(?:e[-+]?\d+)?", s)]
    five = {}
    for m in re.finditer(r"hits\[:, (\d)\] \.= \[([^\]]+)\]", src.split("if n > 3")[0]):
        five.setdefault(int(m.group(1)), vec(m.group(2)))
    five_ge = {}
    for m in re.finditer(r"hits_ge\[:, (\d)\] \.= \[([^\]]+)\]", src):
        five_ge[int(m.group(1))] = vec(m.group(2))
    rest = src.split("if n > 3", 1)[1]
    four = {}
    for m in re.finditer(r"hits\[:, (\d)\] \.= \[([^\]]+)\]", rest.split("else")[0]):
        four[int(m.group(1))] = vec(m.group(2))
    ge_entries = {}
    for m in re.finditer(r"hits_ge\[(\d), (\d)\] = ([-+]?\d*\.\d+(?:e[-+]?\d+)?)", src):
        ge_entries[(int(m.group(1)), int(m.group(2)))] = float(m.group(3))
    fixtures = {}
    fixtures["5"] = {"hits": [five[i] for i in range(1, 6)], "ge": [five_ge[i] for i in range(1, 6)]}
    for n in (3, 4):
        ge = [[0.0] * 6 for _ in range(n)]
        for (r, c), v in ge_entries.items():
            if c <= n:
                ge[c - 1][r - 1] = v
        fixtures[str(n)] = {"hits": [four[i] for i in range(1, n + 1)], "ge": ge}
    b = float(re.search(r"B = ([0-9.]+)", src).group(1))
    return fixtures, b


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of a CMS-Julia checkout (holds src/julia-serial)")
    args = ap.parse_args()
    for kn in range(5):
        i, x, y, a, ncl = generate_clusters(kn)
        np.savez_compressed(HERE / f"clustering_kn{kn}.npz", id=i, x=x, y=y, adc=a, ncl=np.int64(ncl))
        print(f"kn={kn}: {len(i)} digis, {ncl} clusters")
    np.savez_compressed(HERE / "clustering_diag8.npz", id=np.ones(8, np.uint16),
                        x=np.array([1, 3, 5, 7, 9, 11, 13, 2], np.int16),
                        y=np.array([1, 3, 5, 7, 9, 11, 13, 2], np.int16), adc=np.full(8, 5000, np.int32),
                        ncl=np.int64(6))
    fixtures, b = parse_brokenline(Path(args.reference))
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import oracle
    out = {"B": b, "source": "test/testBrokenLine.jl:12-81", "fits": {}}
    for n, fx in fixtures.items():
        hits = np.array(fx["hits"], np.float64).T
        ge = np.array(fx["ge"], np.float32).T
        r = oracle.bl_fit(hits, ge, b)
        out["fits"][n] = {"hits": fx["hits"], "ge": fx["ge"], "oracle": {k: (v.tolist() if hasattr(v, "tolist") else v)
                                                                        for k, v in r.items()}}
        print(n, r["state"], r["pt"], r["chi2_line"], r["chi2_circle"])
    (HERE / "brokenline_fixtures.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
