"""bench.py's bookkeeping on the CPU: the byte models behind the roofline
figures, the arithmetic a form reports, the reference arm's core count, and
one bounded run of the reference arm on a small world."""
import json
import os
import subprocess
import sys

import pytest

import bench
from worldinagrain_b200 import abi


def test_level_byte_models():
    # per level: (down launch cells, up launch cells, coarse kernel's first)
    s = {"levels": [(262144, 262144, 0), (65536, 65536, 0), (16384, 0, 16384)]}
    # down: 180 B a cell averaged over the levels restricted by tile kernels
    assert bench.level_bytes("F_RESTRICT", s) == (180 * 262144 + 180 * 65536 + 180 * 16384) // 3
    # up: 51 B a cell over the levels above the coarse kernel's
    assert bench.level_bytes("F_PROLONG", s) == (51 * 262144 + 51 * 65536) // 2
    # the coarse kernel: 28 B a cell of its first level
    assert bench.level_bytes("F_COARSE", s) == 28 * 16384
    assert bench.level_bytes("F_RELAX", s) is None
    assert bench.level_bytes("F_RESTRICT", {}) is None
    # the mixed form: the operator words of levels 1 down in binary16 and
    # their potentials in bf16, no stored diagonal there; level 0's
    # coefficients from their binary16 copies
    m = dict(s, mixed=True)
    assert bench.level_bytes("F_RESTRICT", m) == (122 * 262144 + 82 * 65536 + 82 * 16384) // 3
    assert bench.level_bytes("F_PROLONG", m) == int(23.5 * 262144 + 23.5 * 65536) // 2
    assert bench.level_bytes("F_COARSE", m) == 14 * 16384


def test_level_stats_follow_the_coarse_kernels_first_level():
    """The level list the byte models average over: the tile kernels' levels
    end where the batch's coarse_cells launch shape starts the coarse
    kernel, per world."""
    from types import SimpleNamespace
    w512 = SimpleNamespace(L=abi.layout_py(512, 512))
    w64 = SimpleNamespace(L=abi.layout_py(64, 64))
    assert bench.level_stats([w512]) == [(65536, 65536, 0), (16384, 16384, 0), (4096, 0, 4096)]
    assert bench.level_stats([w512], 2048) == [(65536, 65536, 0), (16384, 16384, 0), (4096, 4096, 0),
                                                (1024, 0, 1024)]
    # a 64x64 world's coarse kernel starts at its level 1 (1024 cells): the
    # level-1 down launch takes it, the up launch doesn't
    assert bench.level_stats([w512, w64]) == [(65536 + 1024, 65536, 1024), (16384, 16384, 0), (4096, 0, 4096)]
    s = {"levels": bench.level_stats([w512, w64])}
    assert bench.level_bytes("F_COARSE", s) == 28 * (1024 + 4096)


def test_algorithmic_bytes_of_the_cg_kernels():
    s = {"active_cells": 640, "fluid_cells": 512, "particles": 2048, "levels": []}
    assert bench.algorithmic_bytes("F_UPDATE", s) == 640 * 4 + 512 * (16 + 4 + 24)
    assert bench.algorithmic_bytes("F_APPLY_ALPHA", s) == 640 * 12 + 512 * (8 + 4 + 16 + 8 + 1 + 4) + 128 * 8
    assert bench.algorithmic_bytes("NO_SUCH_PASS", s) is None


def test_traffic_scales_the_captured_ratio():
    """roofline.traffic: a captured launch's DRAM bytes per algorithmic byte
    times this launch's algorithmic bytes; none for kernels not captured."""
    alg = 262144 * 180
    t, src = bench.traffic_of("F_RESTRICT", alg)
    assert abs(t - 23.90272e6) < 2 and "k_fDown" in src
    assert bench.traffic_of("F_RESTRICT", alg // 2)[0] == round(t / 2)
    assert bench.traffic_of("F_COARSE", 10 ** 6) == (None, None)
    assert bench.traffic_of("F_RELAX", 0) == (None, None)


def test_launch_overrides():
    assert bench.launch_overrides(["cg_per_sm=8", "coarse_cells=2048"]) == {"cg_per_sm": 8, "coarse_cells": 2048}
    for bad in (["cg=8"], ["cg_per_sm=0"], ["cg_per_sm=x"], ["cg_per_sm"]):
        with pytest.raises(SystemExit):
            bench.launch_overrides(bad)


def test_form_arithmetic():
    assert bench.dtype_of("mixed") == "bf16+f16+f32+f64"
    assert bench.dtype_of("fast") == bench.dtype_of("plain") == "f32+f64"
    assert bench.FLAGS & abi.STEP_TOLERANCE and bench.FLAGS & abi.STEP_F64_DOTS


def test_reference_cores_bounded_by_memory_and_cap():
    n = bench.reference_cores(1)
    assert 1 <= n <= 64
    assert bench.reference_cores(1 << 62) == 1  # no room for a second replica


def test_reference_arm_prints_one_line(tmp_path):
    env = dict(os.environ, PYTHONPATH=bench.ROOT)
    out = subprocess.run([sys.executable, os.path.join(bench.ROOT, "bench.py"), "--impl", "reference", "--config",
                          "dam", "--steps", "1", "--warmup", "1", "--cpu-budget", "1"],
                         capture_output=True, text=True, timeout=600, env=env, cwd=str(tmp_path))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
