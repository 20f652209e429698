"""CPU tests of the C-ABI library: it loads, exports every symbol the public
header declares, and reports argument and file errors without a GPU."""
import ctypes as C
import os
import subprocess

import pytest

import grass_b200 as G


def test_library_exports_every_declared_symbol():
    declared = G.exported_symbols()
    assert len(declared) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing


def test_every_symbol_resolves_via_ctypes():
    for s in G.exported_symbols():
        assert getattr(G.lib, s) is not None


def test_version_and_counters():
    assert b"sm_100a" in G.lib.grass_version()
    assert G.launch_count() >= 0


def test_open_missing_file_is_io_error(tmp_path):
    with pytest.raises(G.GrassError) as e:
        G.Graph(str(tmp_path / "nope"), "GT")
    assert e.value.code == G.E_IO
    assert "Open graph file failed" in str(e.value)


def test_open_bad_mode_and_empty_offset():
    with pytest.raises(G.GrassError) as e:
        G.Graph.from_bytes(b"\x00" * 8, b"\x04\x10", mode=7)
    with pytest.raises(KeyError):
        G.Graph.from_bytes(b"\x00" * 8, b"\x04\x10", mode="XX")
    h = C.c_void_p()
    rc = G.lib.grass_open_mem(None, 0, C.c_char_p(b"\x04"), 1, 0, 0, C.byref(h))
    assert rc == G.E_FORMAT


def test_null_arguments_are_rejected():
    assert G.lib.grass_rw(None, None, None, 0, None, None, None) == G.E_ARG
    assert G.lib.grass_khop(None, None, None, 0, None, None, None) == G.E_ARG
    assert G.lib.grass_get_info(None, None) == G.E_ARG
    assert G.lib.grass_close(None) == G.OK


def test_header_has_citations():
    txt = open(G.INCLUDE).read()
    for ref in ("GT/src/grass.cu", "GT/src/bcg.cuh", "LE/src/bcg.cuh", "compressor.hpp",
                "randomWalks.cu", "khop.cu", "multiRW.cu"):
        assert ref in txt


def test_compaction_arguments_are_checked_before_any_device_work():
    """The edge-list calls reject bad arguments on the host (no GPU needed)."""
    with pytest.raises(G.GrassError) as e:  # no count word
        G.khop_edges_device(None, 0, (25, 10), [None, None], None, None, 0, None)
    assert e.value.code == G.E_ARG
    with pytest.raises(G.GrassError) as e:  # capacity without outputs
        G.rw_edges_device(16, 4, 8, None, None, 4, 16)
    assert e.value.code == G.E_ARG
    with pytest.raises(G.GrassError) as e:  # layout out of range
        G.rw_edges_device(16, 4, 8, None, None, 0, 16, layout=5)
    assert e.value.code == G.E_ARG
    with pytest.raises(G.GrassError) as e:  # zero fanout
        G.khop_edges_device(None, 0, (25, 0), [None, None], None, None, 0, 16)
    assert e.value.code == G.E_ARG
    with pytest.raises(G.GrassError) as e:  # multi-RW steps without step buffers
        G.mrw_edges_device(None, None, 4, 10, None, None, 0, 16)
    assert e.value.code == G.E_ARG
    with pytest.raises(G.GrassError) as e:  # probe size not a power of two
        G.random_read_probe(16, 1000, 10, 1, 16)
    assert e.value.code == G.E_ARG
