"""CLI: the reference's flags and output format (fastesp/cli.py:193-199, 292-301)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle.esp_oracle as O
from fastesp_b200 import cli


def test_points_reader_and_output_format(tmp_path):
    p = tmp_path / "pts.txt"
    p.write_text("# header\n3\n 0.0 1.0 2.0\n1 2\n1.5 -2.5 3.25 extra\nx y z\n")
    pts = cli.read_points(p)
    np.testing.assert_array_equal(pts, [[0.0, 1.0, 2.0], [1.5, -2.5, 3.25]])
    np.testing.assert_allclose(cli.read_points(p, angstrom=True), pts / 0.529177210903)
    out = tmp_path / "esp.txt"
    cli.write_esp(out, pts, np.array([0.125, -1e-3]))
    lines = out.read_text().splitlines()
    assert lines[0] == "2"
    assert lines[1] == f" {0.0:20.12f} {1.0:20.12f} {2.0:20.12f} {0.125:22.14e}"
    back = np.loadtxt(out, skiprows=1)
    np.testing.assert_array_equal(back[:, 3], [0.125, -1e-3])


def test_cpu_backends_are_refused(tmp_path):
    with pytest.raises(SystemExit):
        cli.run_esp(tmp_path / "x.molden", tmp_path / "p.txt", backend="numpy")
    with pytest.raises(SystemExit):
        cli.run_esp(tmp_path / "x.molden", tmp_path / "p.txt", backend="cpp")


def test_selftest_quadrature_is_independent_and_accurate():
    """The selftest's u-integral quadrature against the oracle's McMurchie-Davidson
    integrals: two different methods agreeing to 1e-12."""
    A = np.array([0.3, -0.4, 0.2])
    B = A + np.array([1.1, 0.5, -0.6])
    C = np.array([0.1, 1.6, 1.1])
    for la, lb in [((0, 0, 0), (0, 0, 0)), ((2, 1, 1), (1, 2, 0)), ((2, 2, 0), (0, 2, 2))]:
        r = O.primitive_pair_integral(0.45, A, la, 0.72, B, lb, C)
        q = cli.u_quadrature(0.45, A, la, 0.72, B, lb, C)
        assert abs(q - r) <= 1e-12 * abs(r)


@pytest.mark.gpu
def test_cli_esp_matches_reference_values(tmp_path, small_system):
    from pathlib import Path
    golden_dir = Path(__file__).resolve().parent / "golden"
    wfn, basis, P, g = small_system
    pts = tmp_path / "pts.txt"
    np.savetxt(pts, g["points"], fmt="%.17g")
    out = tmp_path / "esp.txt"
    assert cli.main(["esp", str(golden_dir / "small.molden"), "--points", str(pts), "-o", str(out),
                     "-q"]) == 0
    got = np.loadtxt(out, skiprows=1)
    np.testing.assert_allclose(got[:, 3], g["esp_t12"], rtol=0, atol=1e-12)
    assert cli.main(["selftest", "-q"]) == 0
