"""Pins of the oracle: the C restatement (oracle/port) against the golden
fixtures produced by the reference itself, and the reference build against
its own container test."""
import os
import subprocess

import numpy as np
import pytest

from helpers import (FP64_RTOL, golden_names, highorder_names, lf_of, load, load_highorder, load_stock, nq_of, rel_err,
                     stock_names)
from oracle import REFERENCE_DIR as REF
from oracle import port, ref_driver


@pytest.mark.parametrize("name", golden_names())
def test_port_pattern_matches_reference(name):
    g = load(name)
    Ap, Ai = port.pattern(g["al_ptr"], g["al_dof"].astype(np.int32), int(g["ndof"]))
    assert np.array_equal(Ap, g["Ap"])
    assert np.array_equal(Ai, g["Ai"])


@pytest.mark.parametrize("name", golden_names())
def test_port_values_match_reference(name):
    g = load(name)
    p = g["params"]
    lf, lv = lf_of(g)
    al = (g["al_ptr"], g["al_idx"], g["al_dof"].astype(np.int32), g["al_coef"])
    Ax, rhs = port.assemble(g["xyz"], g["hexes"] - 1, nq_of(g), al, int(g["ndof"]), g["Ap"], g["Ai"],
                            mass=p.get("mass", False), gradcoef=g["gradcoef"] if len(g["gradcoef"]) else None,
                            lf=lf, lf_value=lv)
    assert rel_err(Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(rhs, g["rhs"]) < FP64_RTOL


def test_port_element_matrix_symmetric_and_singular():
    # natural-BC Laplacian element matrix: symmetric, constants in the kernel
    X = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    X = X + 0.05 * np.random.default_rng(0).standard_normal(X.shape)
    idx = [(0 << 19) | (x << 8) | (y << 4) | z for (x, y, z) in
           [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]]
    K = port.element_matrix(X, 3, idx)
    assert np.allclose(K, K.T, atol=1e-14)
    assert np.max(np.abs(K.sum(axis=1))) < 1e-13


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference sources not present")
def test_reference_build_passes_its_container_test():
    subprocess.run(["make", "-C", os.path.join(os.path.dirname(port.HERE), "oracle"), "-s", "REF=" + REF,
                    "judy_test"], check=True, capture_output=True)
    log = open(os.path.join(port.HERE, "_ref", "judy_templates.log")).read()
    assert log.count("OK") >= 61 and "failed" not in log


@pytest.mark.skipif(not ref_driver.available(), reason="reference oracle not built")
def test_reference_driver_reproduces_golden():
    import hermes3d_b200 as h
    g = load("perm_p2_lifting")
    mesh = h.Mesh().set_arrays(g["xyz"], g["hexes"], g["bquads"], g["bmarkers"])
    r = ref_driver.run(mesh, **g["params"])
    assert np.array_equal(r["Ap"], g["Ap"]) and np.array_equal(r["Ai"], g["Ai"])
    assert np.array_equal(r["Ax"], g["Ax"]) and np.array_equal(r["rhs"], g["rhs"])


def test_refmap_fixture_is_consistent():
    """The reference's RefMap dumps (fixture) are self-consistent: irm is the
    transposed inverse of the printed Jacobian matrix (to 6 decimals)."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kat", "refmap_dumps.npz"))
    for name in ["hex1", "hex2", "hex4", "hex8", "hex27"]:
        rm, irm = z[name + "_rm"], z[name + "_irm"]
        prod = np.einsum("eqrc,eqrd->eqcd", irm, rm)      # irm^T rm = I  (irm = J^-T)
        assert np.allclose(prod, np.eye(3), atol=2e-5), name
        assert np.allclose(np.linalg.det(rm), z[name + "_jac"], atol=2e-5), name


@pytest.mark.parametrize("name", highorder_names())
def test_port_matches_reference_at_high_order(name):
    """Orders 5..8 (up to 729 functions, 10^3 points) on jittered elements:
    the restatement's pattern and values against the reference's."""
    g = load_highorder(name)
    p = g["params"]
    lf, lv = lf_of(g)
    al = (g["al_ptr"], g["al_idx"], g["al_dof"].astype(np.int32), g["al_coef"])
    Ap, Ai = port.pattern(g["al_ptr"], g["al_dof"].astype(np.int32), int(g["ndof"]))
    assert np.array_equal(Ap, g["Ap"]) and np.array_equal(Ai, g["Ai"])
    Ax, rhs = port.assemble(g["xyz"], g["hexes"] - 1, nq_of(g), al, int(g["ndof"]), g["Ap"], g["Ai"],
                            mass=p.get("mass", False), gradcoef=g["gradcoef"], lf=lf, lf_value=lv)
    assert rel_err(Ax, g["Ax"]) < FP64_RTOL
    assert rel_err(rhs, g["rhs"]) < FP64_RTOL


@pytest.mark.parametrize("name", stock_names())
def test_port_stock_rule_matches_reference(name):
    """The restatement of the stock per-pair rule against the reference run
    with its stock forms (--qmode ref) on non-affine meshes."""
    g = load_stock(name)
    al = (g["al_ptr"], g["al_idx"], g["al_dof"].astype(np.int32), g["al_coef"])
    lf, lv = lf_of(g)
    gc = g["gradcoef"] if len(g["gradcoef"]) else None
    Ax, rhs = port.assemble_stock(g["xyz"], g["hexes"] - 1, al, int(g["ndof"]), g["Ap"], g["Ai"],
                                  mass=g["params"].get("mass", False), gradcoef=gc, lf=lf, lf_value=lv)
    assert rel_err(Ax, g["Ax"]) < FP64_RTOL and rel_err(rhs, g["rhs"]) < FP64_RTOL

