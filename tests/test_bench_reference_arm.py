"""bench.py's reference arm (the reference built from its sources, run on
the host cores) prints one well-formed JSON line; it needs no GPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_its_line():
    from oracle import ref_driver
    if not ref_driver.available():
        pytest.skip("reference build missing")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["dtype"] == "f64"
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "reference"


def test_c2_slabs_cover_the_mesh_exactly():
    """The reference arm's z-slabs of the C2 mesh: every element exactly once,
    with its own vertex coordinates; cube faces keep their markers, cut faces
    get the natural marker."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    from hermes3d_b200.mesh import unit_cube
    n = 8
    mesh = unit_cube(n, 0.2, 3)
    cuts = [0, 3, 5, 8]
    got = []
    for k0, k1 in zip(cuts[:-1], cuts[1:]):
        s = bench.c2_slab(mesh, k0, k1, n=n)
        assert len(s.hexes) == (k1 - k0) * n * n
        got.append(s.xyz[s.hexes - 1])
        inner = [k for k in (k0, k1) if 0 < k < n]
        assert np.sum(s.bmarkers == bench.SLAB_MARKER) == len(inner) * n * n
        assert len(s.bquads) == 4 * (k1 - k0) * n + 2 * n * n
    assert np.array_equal(np.concatenate(got), mesh.xyz[mesh.hexes - 1])
