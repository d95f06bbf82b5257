"""Checkpointed adjoint of K RK4 steps behind ``torch.autograd.Function``.

The forward model is the FP64 ``rk_4_main`` time loop (time_integ.f90:137-493) with the entropy
viscosity mu_e and the time step dt *frozen* along the trajectory: each step n uses the mu_e_n
and dt_n that the undifferentiated solver produced for it (smart_visc_spectral and adapt_dt_cfl
run in the forward pass, but their outputs are treated as constants).  With LES (flag_les = 1)
the step's SGS viscosity mu_sgs_n (sgs_visc after the previous step) is frozen the same way.  The gradient therefore
is the exact gradient of ``replay`` (the frozen-coefficient map), which is what the dot-product
and finite-difference checks compare against.

Memory: states (rho, q, E, mu_e, dt) are kept every ``checkpoint_every`` steps; the backward
pass re-runs each segment from its checkpoint (bitwise identical, the solver is deterministic)
and applies the hand-written step VJP (sod_rk4_step_vjp) in reverse.  With
``keep_trajectory=True`` the forward pass instead keeps every step's state and its three RK
stage states (22.4 doubles per node and step: 160 MB per step at 32^3, 1.3 GB at 64^3, so
tens of steps fit in the GPU's HBM) and the backward pass is the step VJPs alone.

Precision: the trajectory (forward and re-run) can be the FP64 or the mixed path; the step
VJPs are always the FP64 Jacobian-transpose evaluated at the stored stage states.  For the
mixed trajectory the gradient is therefore that of the FP64 map along the mixed trajectory,
which differs from the exact gradient of the mixed map by the mixed path's rounding
(relative 1e-7 to 1e-6).
"""
from __future__ import annotations

from dataclasses import dataclass

from .solver import FP64, Sod2dMesh, Sod2dState, _torch


@dataclass
class _Ckpt:
    rho: object
    q: object
    E: object
    mu_e: object
    dt: object
    mu_sgs: object = None  # LES: the step's frozen SGS viscosity


def _clone_state(src: Sod2dState) -> Sod2dState:
    dst = Sod2dState(src.npoin, src.nelem)
    for f in Sod2dState.FIELDS:
        getattr(dst, f).copy_(getattr(src, f))
    dst.dt.copy_(src.dt)
    return dst


def _les(mesh: Sod2dMesh) -> bool:
    return int(getattr(mesh.prm, "flag_les", 0)) == 1


def _ckpt(s: Sod2dState, les: bool = False) -> _Ckpt:
    return _Ckpt(s.rho.clone(), s.q.clone(), s.E.clone(), s.mu_e.clone(), s.dt.clone(),
                 s.mu_sgs.clone() if les else None)


def _load(s: Sod2dState, c: _Ckpt):
    s.rho.copy_(c.rho)
    s.q.copy_(c.q)
    s.E.copy_(c.E)
    s.mu_e.copy_(c.mu_e)
    s.dt.copy_(c.dt)
    if c.mu_sgs is not None:
        s.mu_sgs.copy_(c.mu_sgs)


def rollout(mesh: Sod2dMesh, state: Sod2dState, nsteps: int, checkpoint_every: int = 10, precision: int = FP64,
            stages=None, tail=None):
    """Run nsteps steps in place (dt from the CFL condition after every step, as rk_4_main)
    and return the checkpoints [(step index, _Ckpt)] at multiples of checkpoint_every.  With
    stages (nsteps, 15*npoin) every step is a checkpoint and records its stage states there.
    With tail (a list; stages None) the last segment runs with its stage states recorded into a
    buffer of min(checkpoint_every, nsteps) steps, and tail receives [per-step states, buffer]:
    the backward pass then starts without re-running that segment, and reuses the buffer for the
    others (the size it would allocate itself)."""
    torch = _torch()
    ck = []
    les = _les(mesh)
    last = ((nsteps - 1) // checkpoint_every) * checkpoint_every if nsteps > 0 else 0
    buf = stack = None
    if tail is not None and stages is None and nsteps > 0:
        buf = torch.empty(min(checkpoint_every, nsteps), 15 * state.npoin, dtype=torch.float64, device="cuda")
        stack = []
    for n in range(nsteps):
        if stages is not None or n % checkpoint_every == 0:
            ck.append((n, _ckpt(state, les)))
        if stages is not None:
            mesh.rk_4_main_record(state, stages[n], update_dt=True, precision=precision)
        elif buf is not None and n >= last:
            stack.append(_ckpt(state, les))
            mesh.rk_4_main_record(state, buf[n - last], update_dt=True, precision=precision)
        else:
            mesh.rk_4_main(state, precision, update_dt=True)
    if buf is not None:
        tail.extend([stack, buf])
    return ck


def replay(mesh: Sod2dMesh, state: Sod2dState, mu_e_seq, dt_seq, precision: int = FP64, mu_sgs_seq=None):
    """The frozen-coefficient forward map: step n with mu_e_seq[n], dt_seq[n] (device (1,)) and,
    with LES, mu_sgs_seq[n]."""
    for n, (mu_e, dt) in enumerate(zip(mu_e_seq, dt_seq)):
        state.mu_e.copy_(mu_e)
        state.dt.copy_(dt)
        if mu_sgs_seq is not None:
            state.mu_sgs.copy_(mu_sgs_seq[n])
        mesh.rk_4_main(state, precision, update_dt=False)
    return state


def trajectory_coefficients(mesh: Sod2dMesh, state: Sod2dState, nsteps: int, precision: int = FP64,
                            with_sgs: bool = False):
    """(mu_e_n, dt_n) of each step of the unfrozen forward run from a copy of state, and the
    steps' mu_sgs_n as a third list when with_sgs."""
    s = _clone_state(state)
    mus, dts, sgs = [], [], []
    for _ in range(nsteps):
        mus.append(s.mu_e.clone())
        dts.append(s.dt.clone())
        sgs.append(s.mu_sgs.clone())
        mesh.rk_4_main(s, precision, update_dt=True)
    return (mus, dts, sgs) if with_sgs else (mus, dts)


def backward_through(mesh: Sod2dMesh, template: Sod2dState, ckpts, nsteps: int, bar_rho, bar_q, bar_E,
                     store_stages: bool = True, precision: int = FP64, trajectory=None, tail=None):
    """Adjoint of nsteps steps: (bar_rho, bar_q, bar_E) at step nsteps -> at step 0, in place.
    Each segment is re-run from its checkpoint; with store_stages the re-run keeps the RK stage
    states (15*npoin doubles per step) so that the step VJPs need no second recompute.  With
    trajectory (the forward's per-step stage states, every step a checkpoint) nothing is re-run;
    with tail (rollout's record of the last segment) that segment is not re-run."""
    torch = _torch()
    if trajectory is not None:
        for t in range(nsteps - 1, -1, -1):
            cs = ckpts[t][1]
            mesh.rk4_step_vjp(cs.rho, cs.q, cs.E, cs.mu_e, template.mu_factor, cs.dt, bar_rho, bar_q, bar_E,
                              out=(bar_rho, bar_q, bar_E), stages=trajectory[t], mu_sgs=cs.mu_sgs)
        return bar_rho, bar_q, bar_E
    s = _clone_state(template)
    bounds = [c[0] for c in ckpts] + [nsteps]
    longest = max(bounds[i + 1] - bounds[i] for i in range(len(ckpts)))
    use_tail = bool(tail) and store_stages and tail[1].shape[0] >= longest
    if use_tail:
        stages = tail[1]
    else:
        stages = (torch.empty(longest, 15 * s.npoin, dtype=torch.float64, device="cuda") if store_stages else None)
    for seg in range(len(ckpts) - 1, -1, -1):
        n0, c = ckpts[seg]
        n1 = bounds[seg + 1]
        if use_tail and seg == len(ckpts) - 1:
            stack = tail[0]  # the forward pass recorded this segment's states and stage states
        else:
            _load(s, c)
            stack = []
            les = c.mu_sgs is not None
            for t in range(n1 - n0):
                stack.append(_ckpt(s, les))
                if store_stages:
                    mesh.rk_4_main_record(s, stages[t], update_dt=True, precision=precision)
                else:
                    mesh.rk_4_main(s, precision, update_dt=True)
        for t in range(n1 - n0 - 1, -1, -1):
            cs = stack[t]
            mesh.rk4_step_vjp(cs.rho, cs.q, cs.E, cs.mu_e, template.mu_factor, cs.dt, bar_rho, bar_q, bar_E,
                              out=(bar_rho, bar_q, bar_E), stages=stages[t] if store_stages else None,
                              mu_sgs=cs.mu_sgs)
    return bar_rho, bar_q, bar_E


class Sod2dRollout:
    """``Sod2dRollout.apply(mesh, state, rho, q, E, nsteps, checkpoint_every)`` -> (rho_K, q_K, E_K)
    as a differentiable torch function of the initial conserved fields (rho, q, E).
    keep_trajectory: keep every step's stage states from the forward pass (no re-run in the
    backward pass; checkpoint_every and store_stages are then unused)."""

    @staticmethod
    def apply(mesh: Sod2dMesh, state: Sod2dState, rho, q, E, nsteps: int, checkpoint_every: int = 10,
              store_stages: bool = True, precision: int = FP64, keep_trajectory: bool = False):
        torch = _torch()

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, rho_, q_, E_):
                s = _clone_state(state)
                s.rho.copy_(rho_)
                s.q.copy_(q_)
                s.E.copy_(E_)
                s.u.copy_(s.q / s.rho)  # u(pos) of the state (read by slip walls) is q / rho
                traj = (torch.empty(nsteps, 15 * s.npoin, dtype=torch.float64, device="cuda")
                        if keep_trajectory else None)
                tail = [] if (store_stages and not keep_trajectory) else None
                ck = rollout(mesh, s, nsteps, checkpoint_every, precision, stages=traj, tail=tail)
                ctx.ck = ck
                ctx.traj = traj
                ctx.tail = tail
                ctx.template = state
                return s.rho.clone(), s.q.clone(), s.E.clone()

            @staticmethod
            def backward(ctx, g_rho, g_q, g_E):
                z = lambda g, like: torch.zeros_like(like) if g is None else g.contiguous().clone()
                br, bq, bE = z(g_rho, rho), z(g_q, q), z(g_E, E)
                backward_through(mesh, ctx.template, ctx.ck, nsteps, br, bq, bE, store_stages, precision,
                                 trajectory=ctx.traj, tail=ctx.tail)
                ctx.traj = None
                ctx.tail = None
                return br, bq, bE

        return _Fn.apply(rho, q, E)
