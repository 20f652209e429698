"""Register budgets of the kernels whose speed rests on how many blocks stay
resident per SM (CPU only: nvcc cross-compiles and ptxas reports registers).

The memory-waiting kernels carry __launch_bounds__(256, 4), which caps them
at 64 registers.  The LE walk has no cap: at one walker per thread it is
launched as 256-thread blocks, and three stay resident per SM only while it
needs at most 85 registers.  Unbounded kernels drift between builds (a
rebuild of the node2vec kernel once went from 118 to 134 registers and ran
1.9x slower), so a build that pushes the walk past 85 registers fails here
instead of silently losing a third of its warps."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "grass_b200", "csrc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
         "-Xptxas", "-v"]

pytestmark = pytest.mark.skipif(shutil.which("nvcc") is None or shutil.which("c++filt") is None,
                                reason="needs nvcc and c++filt")


def _registers(src, tmp_path):
    """{demangled kernel name: registers} from ptxas -v for one source file."""
    out = subprocess.run(["nvcc", *FLAGS, "-c", os.path.join(CSRC, src), "-o",
                          str(tmp_path / (src + ".o"))], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-2000:]
    regs, name = {}, None
    for line in out.stderr.splitlines():
        m = re.search(r"Function properties for (\S+)", line)
        if m:
            name = m.group(1)
            continue
        m = re.search(r"Used (\d+) registers", line)
        if m and name:
            regs[name] = int(m.group(1))
            name = None
    names = subprocess.run(["c++filt"], input="\n".join(regs), capture_output=True,
                           text=True).stdout.splitlines()
    return dict(zip(names, regs.values()))


def _pick(regs, pattern):
    hits = {k: v for k, v in regs.items() if re.search(pattern, k)}
    assert hits, f"no kernel matches {pattern}"
    return hits


def test_sampler_register_budgets(tmp_path):
    regs = _registers("kernels_sample.cu", tmp_path)
    for k, v in _pick(regs, r"rw_kernel<1, 1>").items():
        assert v <= 85, f"{k}: {v} registers leaves fewer than 3 blocks of 256 per SM"
    for pat in (r"n2v_kernel<[01]>", r"mrw_kernel<[01]>", r"khop_kernel<[01]>"):
        for k, v in _pick(regs, pat).items():
            assert v <= 64, f"{k}: {v} registers"


def test_decode_and_compaction_register_budgets(tmp_path):
    regs = _registers("kernels_decode.cu", tmp_path)
    for k, v in _pick(regs, r"decode_flat_kernel<[01]>").items():
        assert v <= 64, f"{k}: {v} registers"
    regs = _registers("kernels_compact.cu", tmp_path)
    for k, v in _pick(regs, r"compact_fill_kernel<").items():
        assert v <= 64, f"{k}: {v} registers"
