"""The reference's own CUDA evaluator (fastesp/native/esp_gpu.cu, compiled for
sm_100a into oracle/_ref by oracle/Makefile) on tables exported by this
package: same values as the FP64 path here.  Skipped when the binary was not
built (the reference checkout is needed to build it)."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fastesp_b200 import build_table

pytestmark = pytest.mark.gpu
ESP_GPU = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "esp_gpu"


def run_reference_cuda(table, tmp_path, repeats=3):
    pb, out = tmp_path / "pairs.bin", tmp_path / "esp.txt"
    table.write(pb)
    r = subprocess.run([str(ESP_GPU), str(pb), str(out), "--repeats", str(repeats)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    ms = [float(m) for m in re.findall(r"run \d+: ([0-9.]+) ms", r.stdout)]
    return np.loadtxt(out, skiprows=1)[:, 3], min(ms)


@pytest.mark.skipif(not ESP_GPU.exists(), reason="oracle/_ref/esp_gpu not built")
@pytest.mark.parametrize("which", ["small", "frag54"])
def test_reference_cuda_evaluator_agrees(which, request, golden, tmp_path):
    if which == "small":
        wfn, basis, P, g = request.getfixturevalue("small_system")
        pts = g["points"]
    else:
        wfn, basis, P = request.getfixturevalue("frag54")
        pts = golden("frag54_300")["points"]
    tab = build_table(wfn, basis, P, pts)
    ref, ms = run_reference_cuda(tab, tmp_path)
    ours = tab.esp(pts)
    assert np.abs(ref - ours).max() < 1e-10
    print(f"reference esp_gpu: {which} {len(pts)} points, {tab.n_pairs} pairs: {ms:.3f} ms")
