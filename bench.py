"""Benchmark: SOD2D explicit spectral-element RHS (HEX64, p=3) on B200.

Workload: triply periodic [0,2pi]^3 box of 64^3 HEX64 elements
(7,077,888 unique nodes, 5 conserved fields), nodes jittered by a seeded Gaussian
(sigma = 0.05 x GLL node spacing, periodic-consistent), Taylor-Green vortex + seeded
+-1e-3 velocity perturbation, Re=1600, Ma=0.1, entropy viscosity on, dt from CFL 0.5.
A "step" is one explicit RK4 step (4 RHS stages + lumped-mass update + entropy viscosity
+ next dt), timed as K graph-replayed steps.  Metric: Gdof.stage/s = 5*N*4*K / time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 64]

--impl reference times the CPU restatement of the reference loops (the Fortran reference
cannot be built in this image: no Fortran compiler, MPI or HDF5) on all host cores.
Multi-GPU runs are independent replicas (the path has no inter-GPU exchange on one GPU's
scope): value = total node-stages of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RHS Gdof.stage/s (mixed FP32-element/FP64-assembly; FP64 alongside)"
UNIT = "Gdof.stage/s"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _workload(n: int):
    from sod2d_refmap_b200 import mesh as M
    m = M.periodic_box(n, jitter=0.05, seed=1)
    prm = M.TGVParams()
    st = M.taylor_green_state(m, prm, pert_amp=1e-3, seed=0)
    return M, m, prm, st


def _config(n: int, m, extra: dict | None = None) -> dict:
    c = {"workload": f"TGV periodic {n}^3 HEX64 (p=3), jittered 0.05 node spacing, RK4 steps",
         "elements": m.nelem, "nodes": m.npoin, "dofs": 5 * m.npoin, "porder": 3,
         "l2": "inputs larger than L2 (state+geometry > 2 GB vs 126 MB L2)", "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------------------------------
# CPU sample: one RK4 step of the CPU restatement on a slab of element layers of the same mesh
# ------------------------------------------------------------------------------------------
def _slab_oracle(m, prm, st, layers: int):
    """Oracle mesh restricted to the first `layers` element layers in z of mesh m (geometry
    computed by the oracle for those elements, state sliced to their nodes)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from sod2d_refmap_b200 import mesh as M
    n = m.n
    E = n * n * layers
    conn = np.asarray(m.connec[:E], dtype=np.int64)
    nodes, inv = np.unique(conn, return_inverse=True)
    sub = M.BoxMesh(n=n, L=m.L, nelem=E, npoin=len(nodes), npoin_orig=m.npoin_orig,
                    connec=np.asfortranarray(inv.reshape(E, 64).astype(np.int32)),
                    connec_orig=np.asfortranarray(m.connec_orig[:E]), coord=np.asfortranarray(m.coord[nodes]),
                    coord_orig=m.coord_orig, master=m.master, tables=m.tables)
    om = O.OracleMesh(sub, colour=False)
    # colour classes of the slab (parity in x, y, z) so the scatter stays race-free in parallel
    e = np.arange(E)
    ex, ey, ez = e % n, (e // n) % n, e // (n * n)
    col = (ex % 2) + 2 * (ey % 2) + 4 * (ez % 2)
    order = np.argsort(col, kind="stable").astype(np.int32)
    ptrs = np.concatenate([[0], np.cumsum(np.bincount(col, minlength=8))]).astype(np.int32)
    om.cptr, om.celems = ptrs, order
    om.ctx.ncolors = 8
    om.ctx.color_ptr = O.ptr(om.cptr).value
    om.ctx.color_elems = O.ptr(om.celems).value
    s = st.copy()
    for k in ("rho", "E", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid", "mu_factor"):
        setattr(s, k, np.ascontiguousarray(getattr(st, k)[nodes]))
    s.u = np.asfortranarray(st.u[nodes]); s.q = np.asfortranarray(st.q[nodes])
    s.mu_e = np.zeros((E, 64), order="F"); s.mu_sgs = np.zeros((E, 64), order="F")
    return O, om, s


def cpu_sample(m, prm, st, layers: int, reps: int, threads: int):
    """Times `reps` RK4 steps of the oracle on the slab; returns (Gdof.stage/s, seconds, desc)."""
    O, om, s = _slab_oracle(m, prm, st, layers)
    threads = O.set_threads(threads)
    dt = O.adapt_dt(om, s, prm)
    O.rk4(om, prm, s.copy(), dt, 1)  # warm-up
    t0 = time.perf_counter()
    for _ in range(reps):
        O.rk4(om, prm, s, dt, 1)
    sec = time.perf_counter() - t0
    node_stages = 27 * om.nelem * 4 * reps   # 27 unique nodes per element of the periodic box
    desc = (f"{reps} RK4 step(s) of the CPU restatement on a {layers}-layer slab "
            f"({om.nelem} elements = {27 * om.nelem} node-equivalents) of the same mesh")
    return 5 * node_stages / sec / 1e9, sec, desc, threads


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    M, m, prm, st = _workload(args.n)
    layers = args.ref_layers
    O, om, s = _slab_oracle(m, prm, st, layers)
    threads = O.set_threads(os.cpu_count() or 1)
    dt = O.adapt_dt(om, s, prm)
    for _ in range(args.warmup):
        O.rk4(om, prm, s, dt, 1)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.rk4(om, prm, s, dt, 1)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    node_stages = 27 * om.nelem * 4 * args.steps
    value = 5 * node_stages / tot / 1e9
    sample = (f"each step: one RK4 step of the CPU restatement of the reference loops (oracle/, OpenMP, "
              f"{threads} threads) on a {layers}-layer slab ({om.nelem} elements) of the {args.n}^3 mesh")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded TGV on a generated periodic HEX64 mesh)",
            "config": _config(args.n, m, {"sample_elements": om.nelem}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the Fortran/OpenACC reference needs a Fortran compiler, MPI and HDF5, absent here; "
                    "this arm times its line-by-line C++ restatement"}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.5)  # let the sampler start before the timed region
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _rel_l2(a, b):
    a = a.double().flatten(); b = b.double().flatten()
    nb = float(b.norm())
    return float((a - b).norm()) / (nb if nb > 0 else 1.0)


# Arithmetic operations of the reference formulation of one stage RHS (mass, momentum, energy
# residuals incl. EOS, Sutherland, diffusion, convection, assembly and 1/Ml; entropy residual
# not included) per HEX64 element of a periodic mesh (27 unique nodes per element), counted by
# the oracle's operation-counting type (oracle_rhs_opcount; sqrt and pow count as one).
RHS_OPS_PER_ELEMENT = 152800


def fp32_peak_tflops(sm_mhz: float) -> float:
    """Nominal FP32 CUDA-core peak of a B200: 148 SMs x 128 lanes x 2 flops per FMA x clock."""
    return 148 * 128 * 2 * sm_mhz * 1e6 / 1e12


def kr_bytes_per_launch(nelem: int, npoin: int, mixed: bool) -> float:
    """Algorithmic HBM bytes of one fused-RHS launch: per element the geometry (9 He + gpvol),
    mu_e and connectivity read and the 6x64 element residuals written; per node the 5
    conserved fields and mu_factor read once."""
    r = 4 if mixed else 8
    per_elem = 64 * (10 * r + r + 4 + 6 * r)
    per_node = 6 * 8
    return per_elem * nelem + per_node * npoin


def _tune_summary(table):
    """The autotuner's sweep as rows of (elements per CTA, CTAs per SM of the one-launch stage
    or 0 for two launches, ms per stage) and its choice (the fastest row)."""
    best = min(table, key=lambda r: r[2]) if table else None
    return {"columns": ["elements_per_cta", "ctas_per_sm (0: two launches per stage)", "ms_per_stage"],
            "rows": [list(r) for r in table],
            "chosen": None if best is None else {"elements_per_cta": best[0], "ctas_per_sm": best[1]}}


def bench_batch(nmember: int, steps: int):
    """Ensemble of periodic HEX64 boxes, n per side log-uniform in [4, 24]
    (seed 4), Re uniform in [400, 3200] (seed 5), own TGV state and dt; `steps` RK4 steps of
    every member, one launch per stage for the whole ensemble, each step a captured graph.
    Compared with the same members advanced one after another (one graph per member)."""
    import torch
    from sod2d_refmap_b200 import mesh as M, solver as S, _lib
    r4 = np.random.default_rng(4)
    r5 = np.random.default_rng(5)
    ns = np.rint(np.exp(r4.uniform(math.log(4), math.log(24), nmember))).astype(int)
    res = r5.uniform(400.0, 3200.0, nmember)
    prm = M.TGVParams()
    meshes = [M.periodic_box(int(n), jitter=0.05, seed=100 + i) for i, n in enumerate(ns)]
    states = [M.taylor_green_state(m, prm, seed=1000 + i, re=float(re)) for i, (m, re) in enumerate(zip(meshes, res))]
    N = sum(m.npoin for m in meshes)
    E = sum(m.nelem for m in meshes)
    B = S.Sod2dBatch(meshes, states, prm)
    B.adapt_dt()
    dt0 = B.dt()
    out = {"members": nmember, "elements": E, "nodes": N, "steps": steps,
           "n_per_side": {"min": int(ns.min()), "max": int(ns.max()), "mean": float(ns.mean())}}
    out["elements_per_cta"] = {"mixed": B.autotune(S.MIXED)[0], "fp64": B.autotune(S.FP64)[0]}
    out["autotune"] = {name: _tune_summary(B.autotune_table(p)) for p, name in ((S.MIXED, "mixed"), (S.FP64, "fp64"))}
    for prec, name in ((S.MIXED, "mixed"), (S.FP64, "fp64")):
        B.set_dt(dt0)
        B.rk4_steps(3, precision=prec)
        torch.cuda.synchronize()
        l0 = _lib.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B.rk4_steps(steps, precision=prec)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[name] = {"value": 5 * N * 4 * steps / (ms / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms / steps,
                     "launches_per_step": (_lib.launch_count() - l0) / steps}
    B.close()
    # the same members one at a time (each its own mesh, graph and launches)
    total = 0.0
    for m, st in zip(meshes, states):
        gm = S.Sod2dMesh(m, prm)
        s_ = S.Sod2dState.from_host(st, gm.nelem)
        gm.adapt_dt(s_)
        gm.rk4_steps(s_, 1, precision=S.MIXED)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        gm.rk4_steps(s_, steps, precision=S.MIXED)
        e1.record()
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1)
        gm.close()
    out["sequential_mixed"] = {"value": 5 * N * 4 * steps / (total / 1e3) / 1e9, "unit": UNIT,
                               "ms_per_step": total / steps}
    return out


def bench_adjoint(n: int, steps: int, every: int):
    """Adjoint: loss 1/2 ||rho u||^2 after `steps` RK4 steps on an n^3 jittered periodic HEX64
    mesh (seed 3), gradient w.r.t. the initial (rho, q, E) by the checkpointed adjoint
    (checkpoint every `every` steps; mu_e and dt frozen at their forward values), with the
    trajectory in FP64 and in mixed precision (the step VJPs are FP64 in both).  Times the
    forward (with checkpointing) and the backward by CUDA events, and checks the directional
    derivative along a seeded Gaussian direction (seed 9) against central differences of the
    frozen-coefficient forward map of the same precision at h = 1e-4 and 1e-6."""
    import torch
    from sod2d_refmap_b200 import mesh as M, solver as S
    from sod2d_refmap_b200.adjoint import Sod2dRollout, replay, trajectory_coefficients, _clone_state
    m = M.periodic_box(n, jitter=0.05, seed=3)
    prm = M.TGVParams()
    gm = S.Sod2dMesh(m, prm)
    s = S.Sod2dState.from_host(M.taylor_green_state(m, prm), gm.nelem)
    gm.adapt_dt(s)
    gm.rk_4_main(s, S.FP64, update_dt=True)  # a state with mu_e > 0
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    v = [torch.randn(x.shape, dtype=torch.float64, device="cuda", generator=g) * x.abs().mean()
         for x in (s.rho, s.q, s.E)]

    def run(K, prec, keep=False):
        rho = s.rho.clone().requires_grad_(True)
        q = s.q.clone().requires_grad_(True)
        E = s.E.clone().requires_grad_(True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record()
        _, qK, _ = Sod2dRollout.apply(gm, s, rho, q, E, K, every, True, prec, keep)
        loss = 0.5 * (qK * qK).sum()
        ev[1].record()
        loss.backward()
        ev[2].record()
        torch.cuda.synchronize()
        return (rho.grad, q.grad, E.grad), float(loss.item()), ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])

    out = {"mesh": f"{n}^3 HEX64 jittered periodic", "nodes": m.npoin, "steps": steps, "checkpoint_every": every}
    dls = {}
    for prec, name in ((S.FP64, "fp64"), (S.MIXED, "mixed")):
        run(2, prec)  # warm-up
        # the kept trajectory of the full step count is allocated here, outside the timed runs,
        # and the timed kept run follows it directly: it then finds the same cached blocks whole
        # (tensors still held from another run, such as its gradients, can pin part of the
        # trajectory's cached block and send the next request to cudaMalloc inside the timing)
        run(steps, prec, True)
        # the forward keeps every step's stage states in HBM: the backward is the VJPs alone
        grads_k, _, t_fwd_k, t_bwd_k = run(steps, prec, True)
        grads, loss, t_fwd, t_bwd = run(steps, prec)
        keep_equal = all(bool(torch.equal(a, b)) for a, b in zip(grads, grads_k))
        t = _clone_state(s)
        gm.rk4_steps(t, steps, precision=prec)  # captures the graph of this step count
        t = _clone_state(s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        gm.rk4_steps(t, steps, precision=prec)
        e1.record()
        torch.cuda.synchronize()
        t_graph = e0.elapsed_time(e1)
        mus, dts = trajectory_coefficients(gm, s, steps, prec)
        dL = float(sum((gi * vi).sum() for gi, vi in zip(grads, v)).item())
        dls[name] = dL

        def L_at(h, p_map=prec):
            u = _clone_state(s)
            u.rho.add_(h * v[0]); u.q.add_(h * v[1]); u.E.add_(h * v[2])
            replay(gm, u, mus, dts, p_map)
            return 0.5 * float((u.q * u.q).sum().item())
        fd = {}
        for h in (1e-4, 1e-6):
            d = (L_at(h) - L_at(-h)) / (2 * h)
            fd[f"{h:g}"] = {"fd": d, "rel_err": abs(d - dL) / abs(dL)}
        if prec == S.MIXED:
            # the mixed gradient is the FP64 map's gradient along the mixed trajectory: central
            # differences of the FP64 map with the mixed run's frozen mu_e and dt carry no FP32
            # rounding noise, so they test it below the mixed map's noise floor
            for h in (1e-4, 1e-6):
                d = (L_at(h, S.FP64) - L_at(-h, S.FP64)) / (2 * h)
                fd[f"fp64_map_{h:g}"] = {"fd": d, "rel_err": abs(d - dL) / abs(dL)}
        out[name] = {"loss": loss, "directional_derivative": dL, "finite_differences": fd,
                     "ms": {"forward_with_checkpoints": t_fwd, "backward": t_bwd, "forward_plain_graph": t_graph,
                            "forward_keeping_trajectory": t_fwd_k, "backward_from_kept_trajectory": t_bwd_k},
                     "adjoint_over_forward": {"backward/forward_with_checkpoints": t_bwd / t_fwd,
                                              "backward/forward_plain_graph": t_bwd / t_graph,
                                              "kept_trajectory_backward/forward": t_bwd_k / t_fwd_k,
                                              "kept_trajectory_backward/forward_plain_graph": t_bwd_k / t_graph},
                     "kept_trajectory_gradient_bitwise_equal": keep_equal,
                     "kept_trajectory_bytes": steps * (20 * m.npoin + 64 * m.nelem) * 8}
    out["mixed"]["directional_derivative_rel_diff_vs_fp64"] = abs(dls["mixed"] - dls["fp64"]) / abs(dls["fp64"])
    out["note"] = ("step VJPs are FP64 in both; the mixed row differentiates the FP64 map along the mixed "
                   "trajectory, and FP32 rounding noise of the mixed map limits its finite differences")
    gm.close()
    return out


def lap_bytes(nelem: int, npoin: int, w: int = 8) -> int:
    """Bytes one matrix-free Poisson product moves at least: per gauss point the metric (6
    values), the connectivity and node->element indices (2 x int32) and the element residual
    written and read back; per node x read, y written and the gather pointer."""
    return nelem * 64 * (6 * w + 8 + 2 * w) + npoin * (2 * w + 4)


def bench_cg(n: int):
    """Pressure-Poisson Jacobi PCG on an n^3 jittered periodic HEX64 mesh (seed 6),
    zero-mean Gaussian right-hand side (seed 7), stop at ||r|| < 1e-10 ||r0||; FP64 CG and FP32
    inner CG + FP64 refinement, time to solution by CUDA events (assembly excluded)."""
    import torch
    from sod2d_refmap_b200 import mesh as M, solver as S
    m = M.periodic_box(n, jitter=0.05, seed=6)
    gm = S.Sod2dMesh(m, M.TGVParams())
    P = S.Sod2dPoisson(gm)
    rng = np.random.default_rng(7)
    rhs = rng.standard_normal(m.npoin)
    rhs -= rhs.mean()
    b = torch.from_numpy(rhs).cuda()
    out = {"mesh": f"{n}^3 HEX64 jittered periodic", "nodes": m.npoin, "elements": m.nelem, "tol": 1e-10}
    P.solve(b, tol=1e-6)              # warm-up: both paths build their iteration graphs here
    P.solve(b, tol=1e-6, mixed=True)
    sols = {}
    for mixed, name in ((False, "fp64"), (True, "mixed")):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        x, it, rel = P.solve(b, tol=1e-10, mixed=mixed)
        e1.record()
        torch.cuda.synchronize()
        sols[name] = x
        out[name] = {"iterations": it, "final_rel_residual": rel, "seconds": e0.elapsed_time(e1) / 1e3}
    out["mixed"]["rel_l2_vs_fp64"] = float((sols["mixed"] - sols["fp64"]).norm() / sols["fp64"].norm())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        P.apply(b)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 10
    nb = lap_bytes(m.nelem, m.npoin)
    out["matvec_fp64"] = {"ms": ms, "bytes": nb, "GBs": nb / ms / 1e6}
    P.close()
    gm.close()
    return out


def run_profile_case(n: int, pin: str = ""):
    """A short, bounded launch sequence for ncu captures: on an n^3 jittered periodic mesh, per
    precision the configuration (pin "EPB:CTAS", or else the autotuner) and 3 RK4 steps (fused
    RHS, stage gather, entropy viscosity + dt kernels; or the one-launch stage kernel), one
    RK4-step VJP (adjoint kernels) and 5 matrix-free Poisson products (element + gather kernels);
    inputs exceed L2 from n = 24 up.  With a pin, the first launches of each precision are its
    three steps' kernels (the fused RHS of stage 1 is the second launch after the mu_e copy)."""
    import torch
    from sod2d_refmap_b200 import solver as S
    M, m, prm, st = _workload(n)
    gm = S.Sod2dMesh(m, prm)
    for prec in (S.FP64, S.MIXED):
        s = S.Sod2dState.from_host(st, gm.nelem)
        gm.adapt_dt(s)
        if pin:
            epb, ctas = (int(x) for x in pin.split(":"))
            gm.set_rhs_config(prec, epb)
            gm.set_stage_launch(prec, ctas)
        else:
            gm.autotune(s, precision=prec)   # the configuration as the benchmark picks it
        for _ in range(3):
            gm.rk_4_main(s, prec, update_dt=True)
    s = S.Sod2dState.from_host(st, gm.nelem)
    gm.adapt_dt(s)
    gm.rk_4_main(s, S.FP64, update_dt=True)
    bars = (s.rho.clone(), s.q.clone(), s.E.clone())
    gm.rk4_step_vjp(s.rho, s.q, s.E, s.mu_e, s.mu_factor, s.dt, *bars)
    P = S.Sod2dPoisson(gm)
    x = s.rho.clone()
    for _ in range(5):
        P.apply(x)
    torch.cuda.synchronize()
    P.close()
    gm.close()
    print(json.dumps({"profile_case": f"{n}^3", "elements": m.nelem, "nodes": m.npoin}))
    return 0


def max_over_ranks(x: float, world: int, device="cuda") -> float:
    """The maximum of x over all ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput of independent replicas: all ranks' units over the slowest time."""
    return units_per_rank * world / seconds_max


def run_ours(args):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    from sod2d_refmap_b200 import solver as S, _lib
    M, m, prm, st0 = _workload(args.n)
    gm = S.Sod2dMesh(m, prm)
    base = S.Sod2dState.from_host(st0, gm.nelem)
    gm.adapt_dt(base)
    torch.cuda.synchronize()
    dt0 = float(base.dt.item())
    stream = torch.cuda.current_stream()
    N, K, W = m.npoin, args.steps, args.warmup

    def fresh():
        s = S.Sod2dState(gm.npoin, gm.nelem)
        for f in S.Sod2dState.FIELDS + ("dt",):
            getattr(s, f).copy_(getattr(base, f))
        return s

    def barrier():
        if world > 1:
            dist.barrier()

    tuned = {}
    tune_tables = {}
    for prec, name in ((S.FP64, "fp64"), (S.MIXED, "mixed")):
        if args.pin_config:
            # a fixed configuration instead of the autotuner (for profiler runs, whose serialised
            # timing would make the tuner choose differently from a live run)
            epb, ctas = (int(x) for x in args.pin_config.split(":"))
            gm.set_rhs_config(prec, epb)
            gm.set_stage_launch(prec, ctas)
            tuned[name] = (epb, float("nan"))
            tune_tables[name] = {"pinned": True, "rows": [], "chosen": {"elements_per_cta": epb, "ctas_per_sm": ctas}}
            continue
        s = fresh()
        tuned[name] = gm.autotune(s, precision=prec)
        tune_tables[name] = _tune_summary(gm.autotune_table(prec))
    results = {}
    states = {}
    clocks = None
    for prec, name in ((S.FP64, "fp64"), (S.MIXED, "mixed")):
        s = fresh()
        gm.rk4_steps(s, W, precision=prec)          # warm-up (also captures the graph)
        s = fresh()
        torch.cuda.synchronize(); barrier(); torch.cuda.synchronize()
        l0 = _lib.launch_count()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(torch.cuda.current_device()) as cs:
            ev0.record(stream)
            gm.rk4_steps(s, K, precision=prec)
            ev1.record(stream)
            torch.cuda.synchronize()
        barrier(); torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        launches = _lib.launch_count() - l0
        results[name] = dict(ms=max_over_ranks(ms, world), launches=launches)
        states[name] = s
        if name == "mixed":
            clocks = cs.summary()
    # accuracy of the mixed path against the FP64 path after K steps (same start, same dt0)
    acc = {k: _rel_l2(getattr(states["mixed"], k), getattr(states["fp64"], k)) for k in ("rho", "q", "E")}
    # TGV diagnostics (volAvg_EK, visc_dissipationRate) of both states after the K steps
    diag = {}
    for name in ("fp64", "mixed"):
        diag[name] = gm.tgv_diagnostics(states[name], prm.rho0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        gm.tgv_diagnostics(states["mixed"], prm.rho0)
    e1.record(stream)
    torch.cuda.synchronize()
    diag["ms_per_call"] = e0.elapsed_time(e1) / 10
    diag["mixed_rel_diff"] = {k: abs(diag["mixed"][k] - diag["fp64"][k]) / abs(diag["fp64"][k])
                              for k in ("EK", "eps_S", "eps_T")}
    s = fresh()
    r64 = gm.rhs(s, precision=S.FP64)
    r32 = gm.rhs(s, precision=S.MIXED)
    acc_rhs = {k: _rel_l2(r32[k], r64[k]) for k in r64}
    # per-kernel durations (CUDA events on the launching stream, eager steps)
    prof = {}
    for prec, name in ((S.FP64, "fp64"), (S.MIXED, "mixed")):
        s = fresh()
        prof[name] = gm.step_profile(s, 5, precision=prec)
    # end to end through the host-buffer C-ABI call (pinned host arrays, copies in the timed region)
    e2e = None
    if True:
        host = {}
        for f in S.Sod2dState.FIELDS:
            t_ = getattr(base, f)
            h = torch.empty(t_.shape, dtype=torch.float64, pin_memory=True)
            h.copy_(t_)
            host[f] = h.numpy()
        host["Reta"] = None
        host["mu_sgs"] = None  # no LES in this case
        n_e2e = max(3, min(K, 10))
        gm.rk4_main_host(host, dt0, precision=S.MIXED)
        torch.cuda.synchronize(); barrier(); torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        dt = dt0
        for _ in range(n_e2e):
            dt = gm.rk4_main_host(host, dt, precision=S.MIXED, stream=stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        sec = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, world)
        E_ = gm.nelem
        h2d = 8 * (N + 3 * N + N + N) + 8 * 64 * E_ + 8
        d2h = 8 * (N + 3 * N + N + 3 * N + 7 * N) + 8 * 64 * E_ + 8
        e2e = {"value": job_throughput(5 * N * 4 * n_e2e, world, sec) / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": n_e2e, "precision": "mixed",
               "api": "sod_rk4_main_host (host arrays in the reference layouts)"}
    value = job_throughput(5 * N * 4 * K, world, results["mixed"]["ms"] / 1e3) / 1e9
    value64 = job_throughput(5 * N * 4 * K, world, results["fp64"]["ms"] / 1e3) / 1e9
    hbm, peak_kind = _peaks()
    kr_ms = prof["mixed"][0]
    kr_bytes = kr_bytes_per_launch(gm.nelem, N, True)
    achieved = kr_bytes / (kr_ms / 1e3) / 1e9
    kr64_bytes = kr_bytes_per_launch(gm.nelem, N, False)
    roof = {"bound": "hbm", "kernel": f"k_rhs_mixed2<{tuned['mixed'][0]}> (fused element RHS, mixed, packed FP32)",
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else "fallback 6650 GB/s",
            "traffic": None, "bytes_per_launch": kr_bytes, "ms_per_launch": kr_ms,
            "fp64_kernel": {"ms_per_launch": prof["fp64"][0], "bytes_per_launch": kr64_bytes,
                            "achieved_GBs": kr64_bytes / (prof["fp64"][0] / 1e3) / 1e9},
            "arithmetic": {"ops_per_launch": RHS_OPS_PER_ELEMENT * gm.nelem,
                           "achieved_tflops": RHS_OPS_PER_ELEMENT * gm.nelem / (kr_ms / 1e3) / 1e12,
                           "peak_tflops": fp32_peak_tflops(1965.0),
                           "frac": RHS_OPS_PER_ELEMENT * gm.nelem / (kr_ms / 1e3) / 1e12 / fp32_peak_tflops(1965.0),
                           "note": "reference-formulation operation count (oracle) over the measured mixed "
                                   "launch time, against the nominal FP32 CUDA-core peak at 1965 MHz "
                                   "(148 SMs x 128 lanes x 2); no measured FP32 peak exists for this pool"},
            "kernel_ms": {"mixed": {"rhs": prof["mixed"][0], "gather_rk": prof["mixed"][1], "visc_dt": prof["mixed"][2]},
                          "fp64": {"rhs": prof["fp64"][0], "gather_rk": prof["fp64"][1], "visc_dt": prof["fp64"][2]}}}
    tr = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.exists(tr):
        kv = {}
        with open(tr) as f:
            for ln in f:
                if "=" in ln and not ln.lstrip().startswith("#"):
                    k_, v_ = ln.split("=", 1)
                    kv[k_.strip()] = v_.strip()
        per_elem = kv.get("k_rhs_mixed2_bytes_per_element")
        if per_elem:
            roof["traffic"] = float(per_elem) * gm.nelem
            roof["traffic_note"] = ("ncu DRAM bytes per element on the 32^3 profile case, scaled by the "
                                    "element count: " + kv.get("source", ""))
        wf = kv.get("k_rhs_mixed2_shared_wavefronts_per_element")
        if wf:
            # the binding resource of the kernel: one 128-byte shared-memory wavefront per SM clock
            clk = (clocks or {}).get("sm_mhz") or 1965.0
            per_s = float(wf) * gm.nelem / (kr_ms / 1e3)
            peak = 148 * clk * 1e6
            roof["shared_memory"] = {"achieved_Gwavefronts_per_s": per_s / 1e9, "peak_Gwavefronts_per_s": peak / 1e9,
                                     "frac": per_s / peak, "achieved_TBs": per_s * 128 / 1e12,
                                     "note": "ncu shared-memory wavefronts per element (32^3 profile case) x elements "
                                             "over the measured launch time, against 1 wavefront (128 B) per SM "
                                             "clock at the sampled SM clock"}
    cg = None if args.no_cg else bench_cg(args.cg_n)
    batch = None if args.no_batch else bench_batch(args.batch_members, args.batch_steps)
    adjoint = None if args.no_adjoint else bench_adjoint(args.adj_n, args.adj_steps, args.adj_every)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, sec, desc, thr = cpu_sample(m, prm, st0, layers=args.cpu_layers, reps=args.cpu_reps,
                                       threads=os.cpu_count() or 1)
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port", "sample": desc, "seconds": sec}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": results["mixed"]["ms"] / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32-element/f64-assembly",
                "data": "synthetic (seeded TGV on a generated periodic HEX64 mesh)",
                "config": _config(args.n, m, {"dt0": dt0, "elements_per_cta": {k: v[0] for k, v in tuned.items()},
                                              "stage_launch": {k: v["chosen"] for k, v in tune_tables.items()}}),
                "autotune": tune_tables,
                "fp64": {"value": value64, "ms_per_step": results["fp64"]["ms"] / K, "dtype": "f64",
                         "speedup_mixed_over_fp64": value / value64},
                "mixed_rel_l2_vs_fp64": {"state_after_steps": acc, "rhs_stage": acc_rhs},
                "tgv_diagnostics_after_steps": diag,
                "gpu_launches": results["mixed"]["launches"],
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "pressure_cg": cg,
                "ensemble": batch, "adjoint": adjoint}
        print(json.dumps(line), flush=True)
    for s in states.values():
        del s
    gm.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--cpu-layers", type=int, default=4)
    ap.add_argument("--cpu-reps", type=int, default=10)
    ap.add_argument("--ref-layers", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--pin-config", default="", help="EPB:CTAS - elements per CTA and stage launch shape "
                                                     "(CTAS 0: two launches per stage) instead of the autotuner")
    ap.add_argument("--no-cg", action="store_true")
    ap.add_argument("--cg-n", type=int, default=48)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-members", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--profile-case", type=int, default=0,
                    help="run the short ncu launch sequence on an n^3 mesh instead of the benchmark")
    ap.add_argument("--adj-n", type=int, default=32)
    ap.add_argument("--adj-steps", type=int, default=50)
    ap.add_argument("--adj-every", type=int, default=10)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile_case:
        return run_profile_case(args.profile_case, args.pin_config)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
