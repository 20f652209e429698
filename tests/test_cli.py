"""The drop-in binaries rw, khop (alias ks) and mrw: the reference's options
and exit behaviour (appMain, GT/src/main.cu:5-41), its timing lines
(GT/src/grass.cu:2127-2130), and samples equal to the oracle's for the
reference apps' default workloads (one walker / seed / sample per vertex,
GT/src/apps/randomwalk/randomWalks.cu:4-24, GT/src/apps/khop/khop.cu:3-8,
GT/src/apps/multiRW/multiRW.cu:3-16)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_graph

BIN = os.path.join(ROOT, "grass_b200", "bin")
APPS = ("rw", "khop", "ks", "mrw")
TIMING = ("EndToEndTime:", "transferEndToEndTime:", "transferDataTime:", "runSamplingTime:")


@pytest.fixture(scope="module")
def binaries():
    if not all(os.path.exists(os.path.join(BIN, a)) for a in APPS):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "grass_b200", "csrc"),
                               "apps"])
    return {a: os.path.join(BIN, a) for a in APPS}


def run(exe, *args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=300)


@pytest.mark.parametrize("app", APPS)
def test_no_options_prints_usage_and_exits_0(binaries, app):
    r = run(binaries[app])
    assert r.returncode == 0
    assert "-g --graph-file" in r.stdout and "-n --nruns" in r.stdout


@pytest.mark.parametrize("app", APPS)
@pytest.mark.parametrize("args", [("-n", "3"), ("--nruns", "2"), ("-h",), ("--help",)])
def test_without_graph_prints_usage_and_exits_0(binaries, app, args):
    r = run(binaries[app], *args)
    assert r.returncode == 0
    assert "usage" in r.stdout


@pytest.mark.parametrize("app", APPS)
@pytest.mark.parametrize("flag", ["-g", "--graph-file"])
def test_missing_graph_file_exits_nonzero(binaries, app, tmp_path, flag):
    """Deviation: the reference prints "Open graph file failed!" and exits 0."""
    r = run(binaries[app], flag, str(tmp_path / "absent"))
    assert r.returncode != 0
    assert "Open graph file failed!" in r.stderr


def test_unknown_option_exits_nonzero(binaries):
    r = run(binaries["rw"], "--no-such-option")
    assert r.returncode != 0 and "unknown option" in r.stderr


def _timing(stdout):
    vals = {}
    for line in stdout.splitlines():
        for key in TIMING:
            if line.startswith(key):
                vals[key] = float(line.split()[1])
    return vals


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["LE", "GT"])
@pytest.mark.parametrize("flag", ["-g", "--graph-file"])
def test_rw_outputs_equal_oracle(binaries, oracle_mod, tmp_path, mode, flag):
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    prefix = os.path.join(d, mode)
    out = tmp_path / "paths.u32"
    r = run(binaries["rw"], flag, prefix, "-n", "2", "--mode", mode, "--output", str(out))
    assert r.returncode == 0, r.stderr
    t = _timing(r.stdout)
    assert set(t) == set(TIMING) and all(v >= 0 for v in t.values())
    og = oracle_mod.OracleGraph(prefix)
    n = og.n
    ref, e = og.rw(mode, np.arange(n, dtype=np.uint32), 80, 7)
    got = np.fromfile(out, dtype=np.uint32).reshape(n, 81)
    np.testing.assert_array_equal(got, ref)
    assert f"SampledEdges: {2 * e}" in r.stdout  # two runs


@pytest.mark.gpu
@pytest.mark.parametrize("app", ["khop", "ks"])
@pytest.mark.parametrize("mode", ["LE", "GT"])
def test_khop_outputs_equal_oracle(binaries, oracle_mod, tmp_path, app, mode):
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    prefix = os.path.join(d, mode)
    out = tmp_path / "hops.u32"
    r = run(binaries[app], "-g", prefix, "--mode", mode, "--output", str(out))
    assert r.returncode == 0, r.stderr
    assert set(_timing(r.stdout)) == set(TIMING)
    og = oracle_mod.OracleGraph(prefix)
    n = og.n
    refs, _ = og.khop(mode, np.arange(n, dtype=np.uint32), (10, 25), 7)
    got = np.fromfile(out, dtype=np.uint32)
    np.testing.assert_array_equal(got, np.concatenate([x.ravel() for x in refs]))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["LE", "GT"])
def test_mrw_outputs_equal_oracle(binaries, oracle_mod, tmp_path, mode):
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    prefix = os.path.join(d, mode)
    out = tmp_path / "mrw.u32"
    r = run(binaries["mrw"], "-g", prefix, "--mode", mode, "-n", "2", "--output", str(out))
    assert r.returncode == 0, r.stderr
    assert set(_timing(r.stdout)) == set(TIMING)
    og = oracle_mod.OracleGraph(prefix)
    n = og.n
    roots = oracle_mod.mrw_roots(n, n, 80, 7)
    src, dst, _, _ = og.mrw(mode, roots, 100, 7, 0)
    got = np.fromfile(out, dtype=np.uint32).reshape(2, n, 100)
    np.testing.assert_array_equal(got[0], src)
    np.testing.assert_array_equal(got[1], dst)


@pytest.mark.gpu
def test_auto_mode_detects_the_format(binaries):
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    for mode in ("LE", "GT"):
        r = run(binaries["rw"], "-g", os.path.join(d, mode), "--walkers", "10")
        assert r.returncode == 0, r.stderr
        assert f"Format: {mode}," in r.stdout


@pytest.mark.parametrize("args", [(), ("-n", "2"), ("--help",)])
def test_usage_matches_the_reference_binary(binaries, args):
    """Where the reference's own rw app has been built (baseline/_ref/rw_gt,
    from its sources), its usage lines and exit status are ours."""
    ref = os.path.join(ROOT, "baseline", "_ref", "rw_gt")
    if not os.path.exists(ref):
        pytest.skip("reference rw app not built here")
    r_ref, r_ours = run(ref, *args), run(binaries["rw"], *args)
    assert r_ref.returncode == r_ours.returncode == 0
    ref_lines = [ln.rstrip() for ln in r_ref.stdout.splitlines() if ln.strip()]
    ours = [ln.rstrip() for ln in r_ours.stdout.splitlines() if ln.strip()]
    assert ours[:len(ref_lines)] == ref_lines
