"""z-slab partition of one mesh (multi-GPU sharding without communication):
host plans per part, the union of the parts against the whole mesh, and the
N > 1 path as 2-rank gloo process groups on the CPU (assembly numerics by the
restatement oracle; each rank reduces its owned columns into the global
matrix, which must equal the whole-mesh assembly bit for bit)."""
import os
import socket

import numpy as np
import pytest

import hermes3d_b200 as h
from oracle import port


def _problem(n=4, p=2, jitter=0.2, seed=3, orders=None):
    mesh = h.unit_cube(n, jitter, seed)
    mesh.ugh()
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    if orders is not None:
        sp.set_element_orders(orders)
    else:
        sp.set_uniform_order(p)
    sp.assign_dofs()
    return mesh, sp


def _disc(sp, nparts=1, part=0):
    d = h.Discretization()
    d.set_spaces(sp)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v)
    d.set_linear_form(h.int_F_v(-6.0))
    d.set_quadrature(p_plus=2)
    if nparts > 1:
        d.set_partition(nparts, part)
    M, V = h.UMFPackMatrix(), h.UMFPackVector()
    d.create(M, V)
    return d, M, V


@pytest.mark.parametrize("nparts", [2, 3])
@pytest.mark.parametrize("mixed", [False, True])
def test_parts_cover_the_whole_pattern(nparts, mixed):
    orders = np.random.default_rng(1).integers(1, 4, size=(64, 3)) if mixed else None
    mesh, sp = _problem(orders=orders)
    _, Mg, _ = _disc(sp)
    owner = np.zeros(sp.ndof, np.int32)
    for part in range(nparts):
        d, M, _ = _disc(sp, nparts, part)
        info = d.partition()
        owned = info["owned"]
        assert info["owned_dofs"] == owned.sum() and info["slab_elements"] > 0
        owner += owned
        lens = np.diff(M.Ap)
        assert np.all(lens[~owned] == 0)
        for j in np.flatnonzero(owned):
            assert np.array_equal(M.Ai[M.Ap[j]:M.Ap[j + 1]], Mg.Ai[Mg.Ap[j]:Mg.Ap[j + 1]])
    assert np.all(owner == 1)          # every DOF owned by exactly one part


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port_no, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port_no)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh, sp = _problem()
        dg, Mg, _ = _disc(sp)                    # whole-mesh pattern (host only)
        d, M, _ = _disc(sp, world, rank)
        info = d.partition()
        owned, elems = info["owned"], info["elements"]
        # this rank's elements, assembled by the oracle into the global pattern
        ids = np.flatnonzero(elems) + 1
        al_all = port.asmlists_from_space(sp, mesh.num_elements)
        ptr, idx, dof, coef = al_all
        sel = [(idx[ptr[e - 1]:ptr[e]], dof[ptr[e - 1]:ptr[e]], coef[ptr[e - 1]:ptr[e]]) for e in ids]
        p2 = np.concatenate([[0], np.cumsum([len(s[0]) for s in sel])]).astype(np.int64)
        al = (p2, np.concatenate([s[0] for s in sel]), np.concatenate([s[1] for s in sel]).astype(np.int32),
              np.concatenate([s[2] for s in sel]))
        Ax, rhs = port.assemble(mesh.xyz, mesh.hexes[ids - 1] - 1, 4, al, sp.ndof, Mg.Ap, Mg.Ai, mass=True, lf=1,
                                lf_value=-6.0)
        col_owned = np.repeat(owned, np.diff(Mg.Ap))
        ax = torch.from_numpy(np.where(col_owned, Ax, 0.0))
        rv = torch.from_numpy(np.where(owned, rhs, 0.0))
        dist.all_reduce(ax)                    # each entry comes from exactly one rank
        dist.all_reduce(rv)
        cnt = torch.from_numpy(owned.astype(np.int64))
        dist.all_reduce(cnt)
        if rank == 0:
            Axg, rhsg = port.assemble(mesh.xyz, mesh.hexes - 1, 4, al_all, sp.ndof, Mg.Ap, Mg.Ai, mass=True, lf=1,
                                      lf_value=-6.0)
            out.put((bool(torch.all(cnt == 1)), bool(np.array_equal(ax.numpy(), Axg)),
                     bool(np.array_equal(rv.numpy(), rhsg))))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_assembly_equals_whole_mesh():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port_no = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port_no, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert res == (True, True, True)


def _refined_problem(nparts=1, part=0):
    mesh = h.unit_cube(4, 0.15, 7)
    mesh.ugh()
    mesh.refine_elements([6, 22, 27, 43])          # hanging nodes in the interior and at the slab cuts
    sp = h.H1Space(mesh)
    sp.set_bc_values(lambda m, x, y, z: x * x + y * y + z * z)
    orders = np.random.default_rng(4).integers(1, 4, size=(mesh.num_elements, 3))
    sp.set_element_orders(orders)
    sp.assign_dofs()
    return mesh, sp


@pytest.mark.parametrize("nparts", [2, 3])
def test_parts_of_a_refined_mesh_cover_the_whole_pattern(nparts):
    """Refined mesh (hanging nodes) with mixed orders: the parts own every DOF
    once, hold only active elements, and their owned columns are the whole
    mesh's."""
    mesh, sp = _refined_problem()
    _, Mg, _ = _disc(sp)
    owner = np.zeros(sp.ndof, np.int32)
    taken = np.zeros(mesh.num_elements, np.int32)
    for part in range(nparts):
        d, M, _ = _disc(sp, nparts, part)
        info = d.partition()
        owned = info["owned"]
        owner += owned
        taken += info["elements"].astype(np.int32)
        assert np.all(np.diff(M.Ap)[~owned] == 0)
        for j in np.flatnonzero(owned):
            assert np.array_equal(M.Ai[M.Ap[j]:M.Ap[j + 1]], Mg.Ai[Mg.Ap[j]:Mg.Ap[j + 1]])
    assert np.all(owner == 1)
    assert np.all(taken[~mesh.active] == 0) and np.all(taken[mesh.active] >= 1)
