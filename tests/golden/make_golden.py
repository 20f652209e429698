#!/usr/bin/env python3
"""Generates the golden fixtures under tests/golden/ from the REFERENCE itself.

Run here, where the GraSS reference sources are mounted; it needs oracle/_ref
(``make -C oracle ref``: the reference's own graph_sort, GT/LE compressors and
its bcg.cuh decoder compiled for the host).  Outputs (committed):

  graphs/<name>/{GT,LE}.graph|.offset  reference compressor output
  graphs/<name>/adj.npz                adjacency the files encode (rowptr, cols)
  graphs/<name>/meta.json              n, num_edges, n_file, ubl, notes
  config1_sha256.json                  SHA-256 of the reference pipeline's files for
                                       the R-MAT scale-16 / edge-factor-16 graph
  philox_kat.json                      Philox4x32-10 blocks from PyTorch's engine

Every file is checked while it is made: the reference decoder must reproduce
the adjacency for every vertex, in both formats.
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
import grass_b200 as G  # noqa: E402


def write_edges(path, pairs):
    with open(path, "w") as f:
        f.write("".join(f"{int(a)} {int(b)}\n" for a, b in pairs))


def csr_from_pairs(pairs, n):
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    rp = np.zeros(n + 1, np.uint64)
    np.add.at(rp, pairs[:, 0] + 1, 1)
    return np.cumsum(rp).astype(np.uint64), pairs[:, 1].astype(np.uint32)


def check_and_store(name, sorted_txt, notes):
    out = os.path.join(HERE, "graphs", name)
    os.makedirs(out, exist_ok=True)
    pairs = np.loadtxt(sorted_txt, dtype=np.int64).reshape(-1, 2)
    meta = {"name": name, "notes": notes}
    for mode in ("GT", "LE"):
        O.ref_compress(mode, sorted_txt, os.path.join(out, mode))
        g = O.OracleGraph(os.path.join(out, mode))
        n = g.n
        rp, cols = csr_from_pairs(pairs, n)
        rrp, rcols = O.ref_decode_all(mode, g.words(), g.offsets())
        assert np.array_equal(rrp, rp) and np.array_equal(rcols, cols), f"{name}/{mode}: ref decode"
        ob = open(os.path.join(out, mode + ".offset"), "rb").read()
        lens = O.ref_offset_lengths(mode, ob, g.n_file)
        assert np.array_equal(lens[:n], np.diff(g.offsets())), f"{name}/{mode}: offsets"
        assert not lens[n:].any()
        meta[mode] = {"n": n, "n_file": g.n_file, "ubl": g.ubl, "num_edges": int(rp[-1]),
                      "graph_bytes": os.path.getsize(os.path.join(out, mode + ".graph"))}
    np.savez_compressed(os.path.join(out, "adj.npz"), rowptr=rp, cols=cols)
    json.dump(meta, open(os.path.join(out, "meta.json"), "w"), indent=1)
    print(name, meta["GT"], meta["LE"])


def make_rmat(tmp):
    src, dst = G.gen_rmat(10, 8, seed=42)
    write_edges(f"{tmp}/e.txt", zip(src, dst))
    O.ref_graph_sort(f"{tmp}/e.txt", f"{tmp}/s.txt")
    check_and_store("rmat_s10_e8", f"{tmp}/s.txt",
                    "R-MAT scale 10, edge factor 8, .57/.19/.19/.05, seed 42 (grass_gen_rmat), "
                    "reference graph_sort (undirected), reference compressor")


def make_edge_cases(tmp):
    rng = np.random.default_rng(7)
    n = 6000
    rows = {}
    # degrees around every geometry boundary of both formats
    degs = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 15, 16, 17, 24, 25, 26, 35, 36, 37, 48, 49, 50,
            63, 64, 65, 99, 100, 101, 255, 256, 257, 1000, 1023, 1024, 1025, 2500]
    centers = rng.choice(np.arange(200, n - 200), size=len(degs), replace=False)
    for c, d in zip(centers, degs):
        lo, hi = max(0, c - 3 * d - 50), min(n, c + 3 * d + 50)
        pool = np.setdiff1d(np.arange(lo, hi), [c])
        nb = rng.choice(pool, size=min(d, len(pool)), replace=False)
        rows[int(c)] = np.sort(nb)
    rows[0] = np.sort(rng.choice(np.arange(1, 3000), 100, replace=False))        # positive only
    rows[n - 1] = np.sort(rng.choice(np.arange(0, n - 1), 77, replace=False))    # negative only
    rows[1] = np.array([n - 1])                                                  # one far neighbor
    rows[2] = np.array([0, 1, n - 1])                                            # wide gaps
    rows[3] = np.array([4])                                                      # adjacent
    # every other row empty (degree 0) except a sparse sprinkle
    for v in rng.choice(np.arange(4, n - 1), 300, replace=False):
        if int(v) not in rows:
            d = int(rng.integers(1, 6))
            rows[int(v)] = np.sort(rng.choice(np.setdiff1d(np.arange(n), [v]), d, replace=False))
    pairs = [(v, int(u)) for v in sorted(rows) for u in rows[v]]
    write_edges(f"{tmp}/s.txt", pairs)
    check_and_store("edge_cases", f"{tmp}/s.txt",
                    "directed, written straight to the compressor: degrees 0..2500 across every "
                    "sqrt-geometry boundary, positive-only (v=0), negative-only (v=n-1), far "
                    "neighbors, isolated vertices (degree 0)")


def make_hub(tmp):
    rng = np.random.default_rng(11)
    n = 60000
    rows = {5: np.sort(rng.choice(np.arange(6, n), 20000, replace=False)),
            40000: np.sort(rng.choice(np.setdiff1d(np.arange(n), [40000]), 9999, replace=False))}
    for v in rng.choice(np.arange(10, n - 1), 500, replace=False):
        if int(v) not in rows:
            rows[int(v)] = np.sort(rng.choice(np.setdiff1d(np.arange(n), [v]), 3, replace=False))
    pairs = [(v, int(u)) for v in sorted(rows) for u in rows[v]]
    pairs.append((n - 1, 0))
    write_edges(f"{tmp}/s.txt", pairs)
    check_and_store("hub", f"{tmp}/s.txt",
                    "directed: hub of degree 20000 (GT blocks of ~141 gaps) and one of 9999 "
                    "with neighbors on both sides")


def make_tiny(tmp):
    pairs = [(0, 1), (1, 0), (1, 2), (2, 1), (2, 3), (3, 2), (3, 4), (4, 3), (4, 5), (5, 4),
             (5, 6), (6, 5)]
    write_edges(f"{tmp}/s.txt", pairs)
    check_and_store("tiny_path7", f"{tmp}/s.txt",
                    "7-vertex path; .offset byte padding holds a whole zero length field, so the "
                    "reference counts n_file = 8 (phantom vertex); n < 256 (reference "
                    "decode_offset launches 0 blocks)")


def make_config1_hashes(tmp):
    src, dst = G.gen_rmat(16, 16, seed=42)
    write_edges(f"{tmp}/e.txt", zip(src, dst))
    O.ref_graph_sort(f"{tmp}/e.txt", f"{tmp}/s.txt")
    out = {"graph": "R-MAT scale 16, edge factor 16, .57/.19/.19/.05, seed 42 (grass_gen_rmat); "
                    "reference graph_sort (undirected) then reference compressor"}
    pairs = np.loadtxt(f"{tmp}/s.txt", dtype=np.int64).reshape(-1, 2)
    out["n"] = int(pairs.max()) + 1
    out["num_edges"] = int(len(pairs))
    out["sorted_sha256"] = hashlib.sha256(open(f"{tmp}/s.txt", "rb").read()).hexdigest()
    for mode in ("GT", "LE"):
        O.ref_compress(mode, f"{tmp}/s.txt", f"{tmp}/{mode}")
        for ext in ("graph", "offset"):
            b = open(f"{tmp}/{mode}.{ext}", "rb").read()
            out[f"{mode}.{ext}"] = {"bytes": len(b), "sha256": hashlib.sha256(b).hexdigest()}
        g = O.OracleGraph(f"{tmp}/{mode}")
        rp, cols = csr_from_pairs(pairs, g.n)
        rrp, rcols = O.ref_decode_all(mode, g.words(), g.offsets())
        assert np.array_equal(rrp, rp) and np.array_equal(rcols, cols)
    json.dump(out, open(os.path.join(HERE, "config1_sha256.json"), "w"), indent=1)
    print("config1", out["n"], out["num_edges"])


def make_philox_kat(tmp):
    import torch
    inc = os.path.join(os.path.dirname(torch.__file__), "include")
    exe = f"{tmp}/kat"
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", inc, "-o", exe,
                           os.path.join(HERE, "philox_kat.cpp")])
    rng = np.random.default_rng(3)
    cases = [[0, 0, 0, 0, 0, 0], [0xFFFFFFFF] * 6,
             [0xa4093822, 0x299f31d0, 0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
             [7, 0, 0, 0, 0, 0x52570001], [42, 0, 3, 123456, 0, 0x4b480001]]
    cases += rng.integers(0, 2**32, size=(40, 6), dtype=np.uint64).tolist()
    inp = "".join(" ".join(f"{int(x):x}" for x in c) + "\n" for c in cases)
    outp = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout
    kat = []
    for c, line in zip(cases, outp.strip().split("\n")):
        kat.append({"key": [int(c[0]), int(c[1])], "ctr": [int(x) for x in c[2:]],
                    "out": [int(x, 16) for x in line.split()]})
    json.dump({"source": "PyTorch at::Philox4_32 (ATen/core/PhiloxRNGEngine.h), 10 rounds",
               "cases": kat}, open(os.path.join(HERE, "philox_kat.json"), "w"), indent=0)
    print("philox kat", len(kat))


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref missing: run `make -C oracle ref` where the reference is mounted")
    tmp = tempfile.mkdtemp(prefix="grass_golden_")
    try:
        make_tiny(tmp)
        make_edge_cases(tmp)
        make_hub(tmp)
        make_rmat(tmp)
        make_config1_hashes(tmp)
        make_philox_kat(tmp)
    finally:
        shutil.rmtree(tmp)


if __name__ == "__main__":
    main()
