"""Host-side helpers of bench.py, checked on the CPU.

* The Mie-series surface error the benchmark reports for the N = 81920 precision form
  (bench.mie_surface_error, scipy's spherical Bessel functions) equals the oracle's restatement of
  the reference's rigid-sphere series and area-weighted L2 (pinned by the reference's golden Mie
  coefficients in tests/test_oracle.py) to 1e-12, at ka = 2, 10 and 40.
* The CPU reference arm's whole-solve timing runs end to end on a small mesh and reports the same
  metric string as the GPU arm.
"""
import json
import subprocess
import sys

import numpy as np

import bench


def test_mie_surface_error_matches_oracle(oracle):
    nodes, tris = oracle.icosphere(1.0, 3)
    c, _, a = oracle.element_geometry(nodes, tris)
    rng = np.random.default_rng(7)
    for k in (2.0, 10.0, 40.0):
        theta = np.arccos(np.clip(c[:, 2] / np.linalg.norm(c, axis=1), -1.0, 1.0))
        ref = oracle.mie_field(k, 1.0, oracle.suggested_sphere_terms(k), 1.0, theta)
        x = ref * (1.0 + 1e-3 * (rng.standard_normal(ref.shape) + 1j * rng.standard_normal(ref.shape)))
        e_bench = bench.mie_surface_error(x, c, a, k, 1.0)
        e_or = oracle.rigid_sphere_surface_error(x, c, a, k, 1.0)
        assert abs(e_bench - e_or) <= 1e-12 * max(e_or, 1e-300) + 1e-15, (k, e_bench, e_or)


def test_reference_arm_small_mesh(tmp_path):
    out = subprocess.run([sys.executable, bench.__file__, "--impl", "reference", "--level", "2", "--k", "2.0",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["iterations"][0] > 0 and "all 320 rows" in line["cpu_baseline"]["sample"]
