"""Benchmark: hp-FEM hexahedral assembly on B200 (elements/s).

Workload (one "step" = one full assembly): the 64^3 = 262,144-hexahedra unit
cube with interior vertices jittered by U(+-0.2h) (seeded), uniform p=2,
4 Gauss points per direction, grad.grad + mass with f = sin(pi x) sin(pi y)
sin(pi z): full CSC matrix (127,263,527 nonzeros) + RHS, FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value: elements assembled per second, inputs resident in HBM, device time
(CUDA events on the launch stream), max over ranks.  With N > 1 every rank
assembles its own 64^3 subdomain (different seed): weak scaling, no
collective on the data path.  e2e: the same through the C ABI call with host
buffers: per step the vertex coordinates go host->device from pinned memory
and Ax + rhs come back device->host into pinned memory.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ELEM_SIDE = 64
P_ORDER = 2
N_POINTS = 4
METRIC = "hp assembly elements/s (FP64, C2: 64^3 jittered, p=2, 4^3 pts, grad+mass, sin source, full CSC+RHS)"

# the other configurations (parity cases; reported with --workload, never the headline)
WORKLOADS = {
    "c2": dict(side=64, jitter=0.2, p=2, nq=4, mass=True, lf="sin", coef=None,
               desc="C2: 64^3=262144 jittered (+-0.2h) hexahedra, p=2, 4^3 Gauss points, grad.grad+mass, "
                    "f=sin(pi x)sin(pi y)sin(pi z), full CSC+RHS"),
    "c1": dict(side=8, jitter=0.0, p=3, nq=5, mass=False, lf=1.0, coef=None,
               desc="C1: 8^3 unit cube, p=3, 5^3 Gauss points, homogeneous Dirichlet, grad.grad, f=1"),
    "c3": dict(side=32, jitter=0.0, p=(1, 6), nq=None, qplus=2, mass=False, lf=1.0, coef=None, refine=0.10,
               desc="C3: 32^3 hexahedra, 10% of them (3277, seeded) refined by REFT_HEX_XYZ -> 55707 active "
                    "elements with hanging nodes, anisotropic orders p_d ~ U{1..6} per element and direction "
                    "(seeded), p_d+2 Gauss points per direction, grad.grad, f=1, homogeneous Dirichlet; "
                    "mixed-order batched path (kernel classes, constrained-element kernel, persistent CTAs, "
                    "CUDA graph)"),
    "c4": dict(side=16, jitter=0.2, p=8, nq=10, mass=False, lf=None, coef=(0.5, 2.0),
               desc="C4: 16^3 jittered hexahedra, p=8, 10^3 Gauss points, a_e grad.grad, a_e ~ U[0.5,2]"),
    "c5": dict(side=32, jitter=0.2, p=3, nq=5, mass=False, lf=1.0, coef="lognormal",
               desc="C5 forward: 32^3 jittered hexahedra, p=3, 5^3 points, a_e grad.grad with a_e = exp(g_e), "
                    "g_e ~ N(0, 0.5^2), f=1"),
}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every ~2 ms from a thread (the timed regions are tens
    of milliseconds), nvidia-smi as the fallback.  Reads only."""

    REASONS = [(0x8, "hw_slowdown"), (0x40, "hw_thermal_slowdown"), (0x20, "sw_thermal_slowdown"),
               (0x4, "sw_power_cap")]

    def __init__(self, index):
        self.index = index
        self.samples = []            # (sm_mhz, max_mhz, reason bits)
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll_nvml(self):
        nv, h = self.nvml
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while True:
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx,
                                     int(nv.nvmlDeviceGetCurrentClocksThrottleReasons(h))))
            except Exception:
                break
            if self.stop.wait(0.002):
                break

    def __enter__(self):
        try:
            self.nvml = self._handle()
            self.thread = threading.Thread(target=self._poll_nvml, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read_smi(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7 and parts[0].replace(".", "").isdigit():
                bits = sum(b for (b, _), v in zip(self.REASONS, parts[3:7]) if v.lower() == "active")
                self.samples.append((float(parts[0]), float(parts[1]), bits))

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml:
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        import statistics
        bits = 0
        for smp in self.samples:
            bits |= smp[2]
        return {"sm_mhz": statistics.median(smp[0] for smp in self.samples),
                "sm_max_mhz": max(smp[1] for smp in self.samples),
                "reasons": sorted(n for b, n in self.REASONS if bits & b), "samples": len(self.samples),
                "source": "nvml" if self.nvml else "nvidia-smi"}


def build_problem(h, seed, device, side=None, workload="c2", partition=None):
    import numpy as np
    w = WORKLOADS[workload]
    side = w["side"] if side is None else side
    mesh = h.unit_cube(side, w["jitter"], seed)
    mesh.ugh()
    if w.get("refine"):
        nb = mesh.num_elements
        ids = np.sort(np.random.default_rng(2000 + seed).choice(nb, int(round(w["refine"] * nb)), replace=False) + 1)
        mesh.refine_elements(ids)
    sp = h.H1Space(mesh)
    if isinstance(w["p"], tuple):
        lo, hi = w["p"]
        sp.set_element_orders(np.random.default_rng(1000 + seed).integers(lo, hi + 1, size=(mesh.num_elements, 3)))
    else:
        sp.set_uniform_order(w["p"])
    sp.assign_dofs()
    d = h.Discretization(device)
    d.set_spaces(sp)
    coef = None
    if w["coef"] == "lognormal":
        coef = np.exp(np.random.default_rng(seed).normal(0.0, 0.5, mesh.num_elements))
    elif w["coef"] is not None:
        coef = np.random.default_rng(seed).uniform(w["coef"][0], w["coef"][1], mesh.num_elements)
    d.set_bilinear_form(h.int_grad_u_grad_v_plus_u_v if w["mass"] else h.int_grad_u_grad_v, coef)
    d.set_linear_form(None if w["lf"] is None else h.int_F_v(w["lf"]))
    if partition is not None:
        d.set_partition(*partition)
    if w.get("qplus") is not None:
        d.set_quadrature(p_plus=w["qplus"])
    else:
        d.set_quadrature(points=w["nq"])
    d.create()
    return mesh, sp, d


def algorithmic_bytes(nnz, ndof, nv, ne):
    # 8 nnz (Ax written) + 8 ndof (rhs) + 24 nv (coordinates read) + 32 ne (connectivity)
    return 8 * nnz + 8 * ndof + 24 * nv + 32 * ne


# FP64 tensor-core (mma.sync.m16n8k8.f64) rate measured on this pool's B200 by a timed loop of
# independent MMAs (16 warps per SM): the denominator of the DMMA kernel's tensor roofline
DMMA_PEAK_TFLOPS = 37.0


def dmma_flops_per_element(p, nq):
    """Tensor-core FLOPs one element costs in k_assemble_fp64_dm (padding included): per (c, c')
    pair and M tile, the non-zero stage-2 blocks plus KS x NT3 stage-3 MMAs of 2 * 16 * 8 * 8 flops."""
    nx = p + 1
    nb = nx * nx
    mt, nt3, kk = (nb + 15) // 16, (nb + 7) // 8, 4 * nq
    ks = (kk + 7) // 8
    cls = [3, 0, 0, 2, 1, 2, 1, 0, 0]
    fy = [0, 3, 0, 1, 2, 0, 0, 2, 1]
    used = {(cls[k], fy[k]) for k in range(9)}
    nz = sum(1 for a in range(ks) for b in range(ks)
             if any((nu // nq, kq // nq) in used for kq in range(8 * a, min(8 * a + 8, kk))
                    for nu in range(8 * b, min(8 * b + 8, kk))))
    return nx * nx * mt * (nz + ks * nt3) * 2 * 16 * 8 * 8


C3_SAMPLE_SIDE = 8


def cpu_baseline_c3(repeat=1):
    """C3 on a bounded sample: the reference on one host core, 8^3 base
    elements with 10 % refined and orders drawn as in the GPU run."""
    import numpy as np
    from hermes3d_b200.mesh import unit_cube
    from oracle import ref_driver
    if not ref_driver.available():
        return None
    n = C3_SAMPLE_SIDE
    w = WORKLOADS["c3"]
    mesh = unit_cube(n)
    refs = np.sort(np.random.default_rng(2000).choice(n ** 3, int(round(w["refine"] * n ** 3)), replace=False) + 1)
    ids = n ** 3 + 8 * len(refs)
    orders = np.random.default_rng(1000).integers(w["p"][0], w["p"][1] + 1, size=(ids, 3)).astype(np.int32)
    r = ref_driver.run(mesh, orders=orders, qmode="pplus:%d" % w["qplus"], source="one", bc="dirichlet0",
                       refine=[(int(e), 7) for e in refs], repeat=repeat)
    nact = n ** 3 + 7 * len(refs)
    t = r["timing"]["t_assemble_median"]
    return {"value": nact / t, "unit": "elements/s", "cores": 1, "kind": "reference",
            "sample": "%d^3 base elements, %d refined (REFT_HEX_XYZ) -> %d active, orders U{1..6}, p+2 points, "
                      "Discretization::assemble, median of %d" % (n, len(refs), nact, repeat)}


SLAB_MARKER = 7          # the cut faces of a z-slab of the C2 mesh: natural (no Dirichlet row)


def c2_slab(mesh, k0, k1, n=N_ELEM_SIDE):
    """Elements k0 <= k < k1 (z layers) of the structured n^3 C2 mesh as a mesh
    of their own, vertices renumbered.  The cube's faces keep their markers
    (essential); the cut faces get SLAB_MARKER and are natural, so every element
    of the slab does exactly the work it does inside the whole mesh."""
    import numpy as np
    from hermes3d_b200.mesh import Mesh
    layer_v = (n + 1) ** 2
    v0, v1 = k0 * layer_v, (k1 + 1) * layer_v
    hexes = mesh.hexes[k0 * n * n:k1 * n * n] - v0
    keep = np.all((mesh.bquads > v0) & (mesh.bquads <= v1), axis=1)
    bq, bm = [mesh.bquads[keep] - v0], [mesh.bmarkers[keep]]
    b, a = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    a, b = a.ravel(), b.ravel()

    def vid(i, j, k):
        return 1 + i + (n + 1) * (j + (n + 1) * (k - k0))
    for kc in (k0, k1):
        if 0 < kc < n:
            bq.append(np.stack([vid(a, b, kc), vid(a + 1, b, kc), vid(a + 1, b + 1, kc), vid(a, b + 1, kc)], 1))
            bm.append(np.full(len(a), SLAB_MARKER))
    return Mesh().set_arrays(mesh.xyz[v0:v1], hexes, np.concatenate(bq), np.concatenate(bm))


def _ref_slab_cmd(mesh_file, out_file, repeat):
    from oracle import ref_driver
    return [ref_driver.DRIVER, "--mesh", mesh_file, "--out", out_file, "--p", str(P_ORDER), "--qmode",
            "fixed:%d" % N_POINTS, "--mass", "--source", "sin", "--bc", "dirichlet0", "--natural-markers",
            str(SLAB_MARKER), "--repeat", str(repeat)]


def cpu_baseline(repeat=3):
    """The reference (oracle/_ref, built from the reference's sources) on one
    host core, on a bounded sample of the workload itself: two z layers
    (8192 elements) from the middle of the seeded 64^3 C2 mesh."""
    import tempfile
    from hermes3d_b200.mesh import unit_cube
    from oracle import ref_driver
    if not ref_driver.available():
        return None
    k0 = N_ELEM_SIDE // 2 - 1
    with tempfile.TemporaryDirectory() as td:
        mf = os.path.join(td, "m.bin")
        c2_slab(unit_cube(N_ELEM_SIDE, 0.2, 0), k0, k0 + 2).save_bin(mf)
        r = subprocess.run(_ref_slab_cmd(mf, os.path.join(td, "o.bin"), repeat), capture_output=True, text=True,
                           check=True)
    t = json.loads(r.stdout.strip().splitlines()[-1])["t_assemble_median"]
    ne = 2 * N_ELEM_SIDE ** 2
    return {"value": ne / t, "unit": "elements/s", "cores": 1, "kind": "reference",
            "sample": "z layers %d-%d (%d elements) of the seeded 64^3 C2 mesh, cut faces natural, "
                      "Discretization::assemble, median of %d" % (k0, k0 + 1, ne, repeat)}


def run_reference_arm(args):
    """--impl reference: the reference's own CPU assembly of the whole seeded
    64^3 C2 mesh on all host cores.  The mesh is cut into one z-slab per
    process (the union is exactly C2; cut faces natural, so each element does
    the work it does in the whole mesh); every process runs the reference's
    single-threaded Discretization::create + assemble on its slab.  A step is
    one assembly of every slab: its time is the slowest process's median."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from hermes3d_b200.mesh import unit_cube
    from oracle import ref_driver
    if not ref_driver.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference oracle binary oracle/_ref/h3d_ref_driver not built"}))
        return 0
    import tempfile
    n = N_ELEM_SIDE
    nproc = max(1, min(os.cpu_count() or 1, n))
    cuts = [round(i * n / nproc) for i in range(nproc + 1)]
    # bounded: about a minute of assembly per process at the reference's ~3.6e3 elements/s per core
    repeat = max(1, min(args.warmup + args.steps, int(60 * 3600 * nproc / n ** 3)))
    mesh = unit_cube(n, 0.2, 0)
    with tempfile.TemporaryDirectory() as td:
        procs = []
        for c in range(nproc):
            mf = os.path.join(td, "m%d.bin" % c)
            c2_slab(mesh, cuts[c], cuts[c + 1]).save_bin(mf)
        t0 = time.time()
        for c in range(nproc):
            procs.append(subprocess.Popen(_ref_slab_cmd(os.path.join(td, "m%d.bin" % c), os.path.join(td, "o%d.bin" % c),
                                                        repeat), stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
        outs = [p.communicate() for p in procs]
        wall = time.time() - t0
    times = []
    for o, e in outs:
        line = o.strip().splitlines()[-1] if o.strip() else "{}"
        times.append(json.loads(line).get("t_assemble_median", float("nan")))
    t_step = max(times)
    value = n ** 3 / t_step
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "elements/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered unit-cube mesh)", "impl": "reference",
        "config": {"workload": WORKLOADS["c2"]["desc"], "ndof": 2048383, "nnz": 127263527,
                   "processes": nproc, "slabs": "z layers %s" % ",".join("%d-%d" % (cuts[i], cuts[i + 1] - 1)
                                                                         for i in range(nproc))},
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": nproc, "kind": "reference",
                         "sample": "the whole 64^3 C2 mesh as %d z-slabs, one reference process each, median of %d "
                                   "assemblies per process, wall %.1fs" % (nproc, repeat, wall)},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def run_adjoint(args):
    """C5 adjoint: dL_k/dg_{k,e} for 16 coefficient fields (one launch for all
    fields), L_k = lam_k^T K(exp(g_k)) u_k - lam_k^T f(exp(g_k)).  value =
    element-field sensitivities per second (device time); e2e = the same
    through Discretization.adjoint with g, u, lam copied from pinned host
    memory and the gradient copied back every step."""
    import numpy as np
    import torch
    import hermes3d_b200 as h
    from hermes3d_b200 import autograd as hag
    nf = 16
    torch.cuda.set_device(0)
    mesh, sp, d = build_problem(h, seed=0, device=0, side=args.side, workload="c5")
    ne, ndof = mesh.num_elements, d.ndof
    rng = np.random.default_rng(5)
    g = torch.from_numpy(rng.normal(0.0, 0.5, (nf, ne))).cuda()
    u = torch.from_numpy(rng.normal(0.0, 1.0, (nf, ndof))).cuda()
    lam = torch.from_numpy(rng.normal(0.0, 1.0, (nf, ndof))).cuda()
    S = torch.empty(nf, ne, dtype=torch.float64, device="cuda")
    grad = torch.empty_like(S)
    stream = torch.cuda.current_stream()
    for _ in range(max(3, args.warmup)):
        d.adjoint(g, u, lam, S, grad, stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            d.adjoint(g, u, lam, S, grad, stream)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = d.last_launch_count() * args.steps
    # e2e through the public call with host buffers
    gh, uh, lh = g.cpu().pin_memory(), u.cpu().pin_memory(), lam.cpu().pin_memory()
    out = torch.empty(nf, ne, dtype=torch.float64).pin_memory()
    nrep = max(1, args.e2e_steps)
    torch.cuda.synchronize()
    c0 = time.perf_counter()
    for _ in range(nrep):
        _, gr = d.adjoint(gh.cuda(non_blocking=True), uh.cuda(non_blocking=True), lh.cuda(non_blocking=True), S, grad)
        out.copy_(gr, non_blocking=True)
        torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - c0) * 1e3 / nrep
    # forward + backward through the torch.autograd binding, for context: the forward
    # is one matrix-free adjoint launch for all fields (its gradient is the backward's)
    # plus the source vector, assembled on the first call (not timed)
    for rep in range(2):
        gg = g.clone().requires_grad_(True)
        torch.cuda.synchronize()
        c0 = time.perf_counter()
        L = hag.assembly_energy(gg, u, lam, d)
        L.sum().backward()
        torch.cuda.synchronize()
        fb_ms = (time.perf_counter() - c0) * 1e3
    hbm, peak_kind = peaks()
    B = 2 * 8 * nf * ndof + 3 * 8 * nf * ne + 24 * mesh.num_vertices + 32 * ne
    achieved = B / (ms * 1e-3) / 1e9
    print(json.dumps({
        "metric": "hp adjoint element-field sensitivities/s (C5: 32^3 jittered hexahedra, p=3, 5^3 points, "
                  "16 coefficient fields a=exp(g), g~N(0,0.5^2), u,lam~N(0,1))",
        "value": nf * ne / (ms * 1e-3), "unit": "element-field sensitivities/s", "n_gpus": 1, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered unit-cube mesh, seeded fields)",
        "config": {"workload": "C5 adjoint, 16 fields, one launch per step", "ndof": ndof, "elements": ne,
                   "fields": nf, "l2": "inputs larger than L2 (u, lam: %.2f GB)" % (16e-9 * nf * ndof)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind,
                     "algorithmic_bytes_per_step": B},
        "e2e": {"value": nf * ne / (e2e_ms * 1e-3), "unit": "element-field sensitivities/s",
                "h2d_bytes_per_step": 8 * nf * (ne + 2 * ndof), "d2h_bytes_per_step": 8 * nf * ne, "ms_per_step": e2e_ms},
        "forward_backward_ms": fb_ms,
        "cpu_baseline": None, "cpu_baseline_note": "the reference has no adjoint",
        "clocks": clk.summary(),
        "finite": bool(torch.isfinite(grad).all().item()),
    }))
    return 0


def split_c4(args):
    """The metric's comparison -- plain FP64 against the tensor-core split
    precisions at their stated relative error -- on the C4 workload (16^3
    jittered hexahedra, p = 8, 10^3 points, a_e grad.grad, a_e ~ U[0.5, 2]),
    all three timed in this run on the device (CUDA events, inputs resident,
    Ax 15.5 GB > L2) with the clocks sampled.  Errors of each split result
    against the FP64 kernel's matrix on the same plan (that kernel is checked
    against the reference's own assembly at p = 5..8 in the GPU tests)."""
    import torch
    import hermes3d_b200 as h
    t0 = time.time()
    mesh, sp, d = build_problem(h, seed=0, device=0, workload="c4")
    setup = time.time() - t0
    ne, nnz = mesh.num_elements, d.nnz
    steps = max(3, min(args.steps, 10))
    res = {"workload": WORKLOADS["c4"]["desc"], "elements": ne, "nnz": nnz, "steps": steps,
           "warmup": max(3, args.warmup), "setup_s": round(setup, 1),
           "against": "FP64 kernel on the same plan (pinned to the reference's assembly at p = 5..8)"}
    stream = torch.cuda.current_stream()
    A = {}
    for name, prec in [("fp64", h.PREC_FP64), ("tf32x3", h.PREC_TF32X3), ("ozaki", h.PREC_OZAKI)]:
        A[name] = torch.empty(nnz, dtype=torch.float64, device="cuda")
        for _ in range(max(3, args.warmup)):
            d.assemble_device(A[name], None, stream, precision=prec)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk:
            e0.record(stream)
            for _ in range(steps):
                d.assemble_device(A[name], None, stream, precision=prec)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        r = {"elements_per_s": ne / (ms * 1e-3), "ms_per_step": ms, "nnz_per_s": nnz / (ms * 1e-3),
             "gpu_launches_per_step": d.last_launch_count(), "clocks": clk.summary()}
        if name != "fp64":
            diff = A[name] - A["fp64"]
            r["err_max_abs_over_max"] = float(diff.abs().max() / A["fp64"].abs().max())
            r["err_frobenius_rel"] = float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(A["fp64"]))
            r["tolerance"] = 1e-6 if prec == h.PREC_TF32X3 else 1e-12
            r["speedup_vs_fp64"] = res["fp64"]["ms_per_step"] / ms
            del diff, A[name]
            torch.cuda.empty_cache()
        res[name] = r
    del A, d
    torch.cuda.empty_cache()
    return res


def run_sweep(args):
    """Orders p = 1..8 (p+2 points per direction, jittered cube, a_e grad.grad,
    32^3 elements for p <= 4, 16^3 above): elements/s of the FP64 path (the
    kernel the library picks: low-order kernels up to p = 4, the high-order
    kernel above) against the two tensor-core split precisions (3xTF32: the
    batched low-order kernel at p <= 2, the high-order path above; Ozaki: the
    high-order path at every order), with each split result's error
    against the FP64 matrix.  One JSON line; not the headline."""
    import numpy as np
    import torch
    import hermes3d_b200 as h
    torch.cuda.set_device(0)
    rows = []
    for p in [int(x) for x in args.sweep_orders.split(",")]:
        side = args.side or (32 if p <= 4 else 16)
        rec = {"p": p, "elements": side ** 3}
        ref = None
        # 3xTF32 at p <= 2: the batched low-order tensor-core kernel (elements
        # stacked in the MMA tile); above, the high-order tensor-core kernel.
        # FP64 from p = 4 is the FP64 tensor-core (DMMA) kernel; beside it the
        # FP64 FMA kernel (p >= 5)
        variants = [("fp64", h.PREC_FP64, False, {})]
        if p >= 5:
            variants.append(("fp64_fma", h.PREC_FP64, False, {"H3DG_HO_FP64_FMA": "1"}))
        variants += [("tf32x3", h.PREC_TF32X3, p > 2, {}), ("ozaki", h.PREC_OZAKI, True, {})]
        for name, prec, force, env in variants:
            os.environ.update(env)
            if force:
                os.environ["H3DG_FORCE_HIGH_ORDER"] = "1"
            try:
                mesh = h.unit_cube(side, 0.2, 0)
                mesh.ugh()
                sp = h.H1Space(mesh)
                sp.set_uniform_order(p)
                sp.assign_dofs()
                d = h.Discretization(0)
                d.set_spaces(sp)
                d.set_bilinear_form(h.int_grad_u_grad_v, np.random.default_rng(0).uniform(0.5, 2.0, side ** 3))
                d.set_linear_form(None)
                d.set_quadrature(p_plus=2)
                d.create()
            finally:
                os.environ.pop("H3DG_FORCE_HIGH_ORDER", None)
            A = torch.empty(d.nnz, dtype=torch.float64, device="cuda")
            for _ in range(max(3, args.warmup)):
                d.assemble_device(A, None, precision=prec)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                d.assemble_device(A, None, precision=prec)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            for key in env:
                os.environ.pop(key, None)
            rec[name + "_ms"] = ms
            rec[name + "_elements_per_s"] = side ** 3 / (ms * 1e-3)
            rec[name + "_kernel"] = d.last_kernel()
            if ref is None:
                ref = A
            else:
                diff = A - ref
                rec[name + "_err_max_over_max"] = float(diff.abs().max() / ref.abs().max())
                rec[name + "_err_frobenius"] = float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(ref))
                del diff
                rec[name + "_speedup_vs_fp64"] = rec["fp64_ms"] / ms
                del A
            del d
            torch.cuda.empty_cache()
        del ref
        torch.cuda.empty_cache()
        rows.append(rec)
        print(json.dumps(rec), file=sys.stderr, flush=True)
    print(json.dumps({"metric": "hp assembly elements/s by order: FP64 vs split precision (3xTF32 <= 1e-6, "
                                "int8-sliced Ozaki <= 1e-12)", "unit": "elements/s", "n_gpus": 1, "steps": args.steps,
                      "data": "synthetic (jittered unit cube, a_e ~ U[0.5,2], seed 0)", "sweep": rows}))
    return 0


def run_geometry(args):
    """Kernel (a) alone: reference-map geometry (signed determinant, transposed
    inverse Jacobian, physical point: 13 doubles = 104 bytes per point) at the
    C2 workload's 4^3 Gauss points of every element, device time with CUDA
    events, output 1.7 GB (> L2).  Achieved HBM = (written + read bytes) / time
    against the measured copy bandwidth.  One JSON line; not the headline."""
    import torch
    import hermes3d_b200 as h
    torch.cuda.set_device(0)
    mesh, sp, d = build_problem(h, 0, 0, side=args.side, workload="c2")
    ne, nq = mesh.num_elements, WORKLOADS["c2"]["nq"] ** 3
    dev = torch.device("cuda", 0)
    jac = torch.empty(ne * nq, dtype=torch.float64, device=dev)
    irm = torch.empty(9 * ne * nq, dtype=torch.float64, device=dev)
    xyz = torch.empty(3 * ne * nq, dtype=torch.float64, device=dev)
    for _ in range(max(3, args.warmup)):
        d.geometry(jac, irm, xyz)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        d.geometry(jac, irm, xyz)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    written = 104 * ne * nq
    read = 24 * (len(mesh.xyz)) + 32 * ne + 4 * ne       # coordinates, connectivity, element ids
    peak, src = peaks()
    achieved = (written + read) / (ms * 1e-3) / 1e9
    print(json.dumps({"metric": "geometry kernel (a): points/s and HBM GB/s", "value": ne * nq / (ms * 1e-3),
                      "unit": "points/s", "n_gpus": 1, "steps": args.steps, "ms_per_step": ms,
                      "config": {"workload": WORKLOADS["c2"]["desc"], "points_per_element": nq, "elements": ne},
                      "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                   "frac": achieved / peak, "bytes_per_step": written + read,
                                   "peak_source": src}}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-split", action="store_true",
                    help="leave out the C4 split-precision object of the default (C2) line")
    ap.add_argument("--side", type=int, default=None, help="elements per cube side (profiling runs only)")
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--partition", action="store_true",
                    help="N > 1: one mesh cut into N z-slab parts (strong scaling) instead of one subdomain per GPU")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "tf32x3", "ozaki"],
                    help="tf32x3 / ozaki: split precision on tcgen05 (3xTF32, or int8 slices with FP64 accuracy); "
                         "high-order path")
    ap.add_argument("--adjoint", action="store_true", help="C5 adjoint line (16 fields) instead of an assembly line")
    ap.add_argument("--sweep", action="store_true", help="orders 1..8: FP64 against both split precisions")
    ap.add_argument("--sweep-orders", default="1,2,3,4,5,6,7,8", help="orders of --sweep")
    ap.add_argument("--geometry", action="store_true", help="geometry kernel (a) alone on the C2 mesh: HBM GB/s")
    args = ap.parse_args()
    if args.geometry:
        return run_geometry(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.adjoint:
        return run_adjoint(args)
    if args.sweep:
        return run_sweep(args)

    import numpy as np
    import torch
    import torch.distributed as dist

    import hermes3d_b200 as h

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    t_setup = time.time()
    part = (world, rank) if args.partition and world > 1 else None
    mesh, sp, d = build_problem(h, seed=0 if part else rank, device=local, side=args.side, workload=args.workload,
                                partition=part)
    t_setup = time.time() - t_setup
    ne, ndof, nnz, nv = mesh.num_active_elements, d.ndof, d.nnz, mesh.num_vertices
    elems_here, nnz_job = ne, world * nnz
    if part:
        pinfo = d.partition()
        elems_here = pinfo["slab_elements"] + pinfo["halo_elements"]
        tn = torch.tensor([nnz], dtype=torch.int64, device="cuda")
        dist.all_reduce(tn)
        nnz_job = int(tn.item())
    prec = {"fp64": h.PREC_FP64, "tf32x3": h.PREC_TF32X3, "ozaki": h.PREC_OZAKI}[args.precision]
    stream = torch.cuda.current_stream()
    Ax = torch.empty(nnz, dtype=torch.float64, device="cuda")
    rhs = torch.empty(ndof, dtype=torch.float64, device="cuda")

    for _ in range(max(3, args.warmup)):
        d.assemble_device(Ax, rhs, stream, precision=prec)
    torch.cuda.synchronize()
    launches_per_step = d.last_launch_count()

    d.enable_kernel_timing(args.steps)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            d.assemble_device(Ax, rhs, stream, precision=prec)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    kt = d.kernel_times()
    kernel_ms = float(np.mean(kt)) if kt else None
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    ms_per_step = ms_max / args.steps
    # partition: the whole mesh is the job (each rank's plan holds its slab + halo)
    job_elements = ne if part else world * ne
    value = job_elements / (ms_per_step * 1e-3)

    # ---- e2e through the C ABI with pinned host buffers
    e2e_value, e2e_ms, ok = None, None, True
    if args.e2e_steps > 0:
        xyz_pin = torch.from_numpy(np.ascontiguousarray(mesh.xyz)).pin_memory()
        Ax_pin = torch.empty(nnz, dtype=torch.float64).pin_memory()
        rhs_pin = torch.empty(ndof, dtype=torch.float64).pin_memory()
        xyz_np, Ax_np, rhs_np = xyz_pin.numpy(), Ax_pin.numpy(), rhs_pin.numpy()
        M, V = h.UMFPackMatrix(), h.UMFPackVector()
        M.Ax, V.v = Ax_np, rhs_np
        d.update_vertices(xyz_np)
        d.assemble(M, V, precision=prec)
        barrier()
        torch.cuda.synchronize()
        c0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            d.update_vertices(xyz_np)
            d.assemble(M, V, precision=prec)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - c0) / args.e2e_steps
        te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e_value = job_elements / float(te.item())
        e2e_ms = 1e3 * float(te.item())
        ok = bool(np.all(np.isfinite(Ax_np))) and bool(np.all(np.isfinite(rhs_np)))
    else:
        ok = bool(torch.isfinite(Ax).all().item())

    # ---- split precision: error of the timed result against the FP64 kernel
    split_error = None
    if prec != h.PREC_FP64:
        d.assemble_device(Ax, rhs, stream, precision=prec)
        A64 = torch.empty_like(Ax)
        d.assemble_device(A64, None, stream)
        torch.cuda.synchronize()
        diff = (Ax - A64)
        split_error = {
            "max_abs_over_max": float(diff.abs().max() / A64.abs().max()),
            "frobenius_rel": float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(A64)),
            "tolerance": 1e-6 if prec == h.PREC_TF32X3 else 1e-12,
            "against": "FP64 kernel on the same plan (itself oracle-checked at 1e-12)"}
        del diff, A64

    if rank == 0:
        hbm, peak_kind = peaks()
        B = algorithmic_bytes(nnz, ndof, nv, ne)
        kms = kernel_ms if kernel_ms else ms_per_step
        achieved = B / (kms * 1e-3) / 1e9
        traffic = None
        kern = {"c2": "assemble_fp64", "c3": "assemble_fp64_mixed", "c1": "assemble_fp64", "c5": "assemble_fp64",
                "c4": {h.PREC_FP64: "assemble_fp64_ho", h.PREC_TF32X3: "assemble_ho_tc",
                       h.PREC_OZAKI: "assemble_ho_oz"}[prec]}[args.workload]
        tf = os.path.join(ROOT, "profiles", "traffic_%s_%s.json" % (args.workload, kern))
        if os.path.exists(tf):
            try:
                traffic = json.load(open(tf)).get("bytes_per_step")
            except Exception:
                traffic = None
        metric = METRIC if args.workload == "c2" else METRIC.replace("C2: 64^3 jittered, p=2, 4^3 pts, grad+mass, sin source",
                                                                        WORKLOADS[args.workload]["desc"])
        if prec == h.PREC_TF32X3:
            metric = metric.replace("(FP64, ", "(split precision 3xTF32 on tcgen05, FP64 geometry/scatter, ")
        elif prec == h.PREC_OZAKI:
            metric = metric.replace("(FP64, ", "(FP64-accurate split: int8-sliced x stage on tcgen05, FP64 elsewhere, ")
        out = {
            "metric": metric,
            "value": value, "unit": "elements/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if part else "weak",
            "vs_baseline": None, "dtype": {h.PREC_FP64: "f64", h.PREC_TF32X3: "tf32x3 (x stage) + f32 (z, y stages) + f64",
                      h.PREC_OZAKI: "int8 x7 slices, int32 accumulate (x stage) + f64"}[prec], "data": "synthetic (seeded jittered unit-cube mesh)",
            "config": {"workload": WORKLOADS[args.workload]["desc"] if args.side in (None, WORKLOADS[args.workload]["side"])
                       else "%s forms on %d^3 elements (profiling size)" % (args.workload.upper(), args.side),
                       "ndof": ndof, "nnz": nnz, "elements_per_gpu": elems_here,
                       "l2": "inputs larger than L2 (Ax alone %.2f GB)" % (8e-9 * nnz),
                       "parallelism": ("z-slab partition of one mesh into %d parts (halo elements replicated, owned "
                                       "columns only, no data-path collective)" % world) if part else
                                      ("replicas: one subdomain per GPU" if world > 1 else "single GPU"),
                       "setup_s": round(t_setup, 2)},
            "nnz_per_s": nnz_job / (ms_per_step * 1e-3),
            "kernel_ms_per_step": kernel_ms,
            "autotuned_variant": d.tuning(),
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind,
                         "algorithmic_bytes_per_step": B},
            "e2e": None if e2e_value is None else {
                "value": e2e_value, "unit": "elements/s", "h2d_bytes_per_step": 24 * nv,
                "d2h_bytes_per_step": 8 * nnz + 8 * ndof, "ms_per_step": e2e_ms},
            "clocks": clk.summary(),
            "finite": ok,
        }
        if d.last_kernel() == "ho_fp64_dmma" and not isinstance(WORKLOADS[args.workload]["p"], tuple):
            # the FP64 tensor-core kernel: its executed MMA flops against the measured DMMA rate
            w = WORKLOADS[args.workload]
            fl = dmma_flops_per_element(w["p"], w["nq"])
            ach = ne * fl / (kms * 1e-3) / 1e12
            out["roofline"]["dmma"] = {"bound": "tensor", "achieved": ach, "peak": DMMA_PEAK_TFLOPS, "unit": "TFLOP/s",
                                       "frac": ach / DMMA_PEAK_TFLOPS, "flops_per_element": fl,
                                       "peak_source": "measured (timed mma.sync.m16n8k8.f64 loop on this B200 pool)"}
        if split_error is not None:
            out["split_error"] = split_error
        if not args.no_cpu_baseline and world == 1 and args.workload in ("c2", "c3") and args.side is None:
            try:
                out["cpu_baseline"] = cpu_baseline() if args.workload == "c2" else cpu_baseline_c3()
            except Exception as ex:  # report, do not fail the GPU number
                out["cpu_baseline"] = {"error": str(ex)[:200]}
    if rank == 0 and world == 1 and args.workload == "c2" and args.side is None and not args.no_split:
        # the metric's other half: plain FP64 against the split precisions on the C4 workload
        del Ax, rhs, d
        torch.cuda.empty_cache()
        out["split"] = split_c4(args)
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
