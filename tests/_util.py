import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def t2n(t):
    """torch tensor in the (3,npoin)/(64,nelem) storage -> numpy in the reference Fortran shape."""
    a = t.detach().cpu().numpy()
    return np.asfortranarray(a.T) if a.ndim == 2 else a


def oracle_bc_map(oracle, bnd):
    """(rho, q, E) -> the same after temporary_bc_routine_dirichlet_prim (mod_bc_routines.f90),
    on copies; the routine's aux_u / aux_p outputs are dropped."""
    def B(rho, q, E):
        r = np.array(rho, dtype=np.float64, copy=True)
        qq = np.array(q, dtype=np.float64, order="F", copy=True)
        e = np.array(E, dtype=np.float64, copy=True)
        u = np.zeros((len(r), 3), order="F")
        pr = np.zeros(len(r))
        oracle.bc_dirichlet_prim(bnd, r, qq, u, pr, e)
        return r, qq, e
    return B


def oracle_bc_jvp_map(oracle, bnd):
    """(y, v, u, du) -> (B(y), J_B v) for the routine in dual numbers, u / du the aux_u the slip
    branch reads and its tangent."""
    def J(y, v, u=None, du=None):
        return oracle.bc_jvp(bnd, y[0], y[1], y[2], v[0], v[1], v[2], u=u, du=du)
    return J


def oracle_step_jvp(oracle, om, prm, st, dt, v, mu_sgs=None, bc=None, bc_jvp=None, wall=None):
    """One rk_4_main step (time_integ.f90:288-426) from the FlowState st and its JVP along
    v = (drho, dq (npoin,3), dE), composed from the oracle's dual-number stage JVPs with mu_e
    (and mu_sgs) frozen.  bc (oracle_bc_map) selects the non-periodic path: the routine on every
    stage state (time_integ.f90:255-259) and on the update (:434-438), with the tangent
    B(y + v) - B(y), exact up to rounding for the affine routines of the wall and passive codes;
    bc_jvp (oracle_bc_jvp_map) takes the routine's tangent from dual numbers instead, with the
    velocity the slip branch reads carried along."""
    def with_state(rho, q, E):
        s = st.copy()
        s.rho = np.ascontiguousarray(rho); s.q = np.asfortranarray(q); s.E = np.ascontiguousarray(E)
        return s

    # the velocity the slip branch reads: zero at stage 1, then q/rho of the previous post-routine
    # stage state, and q/rho of y0 for the update (time_integ.f90:208, 266-285)
    uread = [None, None]

    def vel(y, w):
        u = np.asfortranarray(y[1] / y[0][:, None])
        du = np.asfortranarray((w[1] - u * w[0][:, None]) / y[0][:, None])
        return u, du

    def bmap(y, w):
        if bc_jvp is not None:
            out = bc_jvp(tuple(y), tuple(w), uread[0], uread[1])
            uread[0], uread[1] = vel(*out)
            return out
        if bc is None:
            return tuple(y), tuple(w)
        by = bc(*y)
        byw = bc(*(y[f] + w[f] for f in range(3)))
        return by, tuple(byw[f] - by[f] for f in range(3))
    y0 = (st.rho, st.q, st.E)
    acc_y = [a.copy() for a in y0]
    acc_v = [a.copy() for a in v]
    ys, vs = bmap(y0, v)
    a_next = [0.5, 0.5, 1.0, None]
    b = [1 / 6, 1 / 3, 1 / 3, 1 / 6]
    for s in range(4):
        R, dR = oracle.rhs_jvp(om, prm, with_state(*ys), vs[0], vs[1], vs[2], mu_sgs=mu_sgs, wall=wall)
        Rc = (R[0], np.asfortranarray(R[1:4].T), R[4])
        dRc = (dR[0], np.asfortranarray(dR[1:4].T), dR[4])
        for f in range(3):
            acc_y[f] = acc_y[f] - dt * b[s] * Rc[f]
            acc_v[f] = acc_v[f] - dt * b[s] * dRc[f]
        if a_next[s] is not None:
            ys, vs = bmap(tuple(y0[f] - dt * a_next[s] * Rc[f] for f in range(3)),
                          tuple(v[f] - dt * a_next[s] * dRc[f] for f in range(3)))
    if bc is not None or bc_jvp is not None:
        uread[0], uread[1] = vel(y0, v)
        acc_y, acc_v = (list(t) for t in bmap(acc_y, acc_v))
    return acc_y, acc_v


def slab_oracle(oracle, M, m, layers):
    """The oracle on the first `layers` element layers in z of the periodic box m: returns the
    oracle mesh, the slab's global node ids (slab-local id -> global id), its element count and
    the slab-local ids of the nodes whose elements all lie in the slab."""
    n = m.n
    E = n * n * layers
    conn = np.asarray(m.connec[:E], dtype=np.int64)
    nodes, inv = np.unique(conn, return_inverse=True)
    sub = M.BoxMesh(n=n, L=m.L, nelem=E, npoin=len(nodes), npoin_orig=m.npoin_orig,
                    connec=np.asfortranarray(inv.reshape(E, 64).astype(np.int32)),
                    connec_orig=np.asfortranarray(m.connec_orig[:E]), coord=np.asfortranarray(m.coord[nodes]),
                    coord_orig=m.coord_orig, master=m.master, tables=m.tables)
    om = oracle.OracleMesh(sub, colour=False)
    # race-free parallel scatter: colour classes by element parity in x, y, z
    e = np.arange(E)
    col = (e % n % 2) + 2 * ((e // n) % n % 2) + 4 * ((e // (n * n)) % 2)
    om.cptr = np.concatenate([[0], np.cumsum(np.bincount(col, minlength=8))]).astype(np.int32)
    om.celems = np.argsort(col, kind="stable").astype(np.int32)
    om.ctx.ncolors = 8
    om.ctx.color_ptr = oracle.ptr(om.cptr).value
    om.ctx.color_elems = oracle.ptr(om.celems).value
    mm = 3 * n
    kplane = nodes // (mm * mm)
    interior = np.flatnonzero((kplane >= 1) & (kplane <= 3 * layers - 1))
    return om, nodes, E, interior


def slab_state(st, nodes, E, mu_e=None):
    s = st.copy()
    for k in ("rho", "E", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid", "mu_factor"):
        setattr(s, k, np.ascontiguousarray(getattr(st, k)[nodes]))
    s.u = np.asfortranarray(st.u[nodes])
    s.q = np.asfortranarray(st.q[nodes])
    s.mu_e = np.asfortranarray(np.zeros((E, 64)) if mu_e is None else mu_e[:E])
    s.mu_sgs = np.zeros((E, 64), order="F")
    return s
