"""Plain FP64 PyTorch transcription of the unsplit 2D step for
variable-coefficient acoustics (test infrastructure).

Same operations, in the same order, as step2.f90 / flux2.f90 / limiter.f90 /
philim.f90 with the vc-acoustics Riemann solvers of the oracle, written with
whole-grid tensor slices so that torch.autograd can differentiate it.  Used
(1) as a second oracle for the forward step and (2) as the reference gradient
for the hand-written adjoint (autograd differentiates the branch actually
taken by max/min/where, i.e. with the limiter branches frozen).

Arrays are ghosted and indexed [m, i, j] with padded indices (ghost width 2).
"""
import torch

G = 2


def fill_bcs(a, bcl, bcu, negate):
    """Solver.apply_q_bcs / apply_aux_bcs (src/pyclaw/solver.py:299-576) for
    extrap (1), periodic (2) and wall (3): x then y, lower then upper side,
    written out-of-place so that autograd folds ghost-cell gradients back onto
    the interior cells they were copied from."""
    for d in range(2):
        ax = d + 1
        n = a.shape[ax]
        for upper, bc in ((False, bcl[d]), (True, bcu[d])):
            for gi in range(G):
                if not upper:
                    dst = gi
                    src = {1: G, 2: n - 2 * G + gi, 3: 2 * G - 1 - gi}[bc]
                else:
                    dst = n - 1 - gi
                    src = {1: n - G - 1, 2: 2 * G - 1 - gi, 3: n - 2 * G + gi}[bc]
                val = a.narrow(ax, src, 1)
                if bc == 3 and negate:
                    sign = torch.ones((a.shape[0], 1, 1), dtype=a.dtype)
                    sign[d + 1] = -1.0
                    val = val * sign
                a = a.index_copy(ax, torch.tensor([dst]), val)
    return a


# When a list, every philim call appends (method, r) so that a test can check
# that two evaluations took the same limiter branches.
BRANCH_LOG = None


def branch_ids(r, meth):
    """Index of the philim branch taken for each r (the comparisons of philim)."""
    if meth == 4:
        c = (1.0 + r) / 2.0
        t = torch.where(c < 2.0, c, torch.full_like(c, 2.0))
        b = torch.where(c < 2.0, 1, 2)
        b = torch.where(t < 2.0 * r, b, 3)
        t = torch.where(t < 2.0 * r, t, 2.0 * r)
        return torch.where(0.0 > t, 0, b)
    if meth == 2:
        t = torch.where(1.0 < 2.0 * r, torch.ones_like(r), 2.0 * r)
        b = torch.where(1.0 < 2.0 * r, 1, 2)
        u = torch.where(2.0 < r, torch.full_like(r, 2.0), r)
        bu = torch.where(2.0 < r, 3, 4)
        b = torch.where(t > u, b, bu)
        t = torch.where(t > u, t, u)
        return torch.where(0.0 > t, 0, b)
    if meth == 3:
        return torch.sign(r).to(torch.int64)
    if meth == 5:
        return torch.zeros_like(r, dtype=torch.int64)
    return torch.where(0.0 > torch.where(1.0 < r, torch.ones_like(r), r), 0, torch.where(1.0 < r, 1, 2))


class _Ratio(torch.autograd.Function):
    """r = b / a with the derivative written as (g/a, -(g/a) r): torch's own
    division backward forms b / (a*a), which underflows to a division by zero
    when a (a squared wave norm) is subnormal."""

    @staticmethod
    def forward(ctx, b, a):
        r = b / a
        ctx.save_for_backward(a, r)
        return r

    @staticmethod
    def backward(ctx, g):
        a, r = ctx.saved_tensors
        ga = g / a
        return ga, -ga * r


def philim(a, b, meth):
    r = _Ratio.apply(b, a)
    if BRANCH_LOG is not None:
        BRANCH_LOG.append(branch_ids(r.detach(), meth))
    if meth == 4:
        c = (1.0 + r) / 2.0
        t = torch.where(c < 2.0, c, torch.full_like(c, 2.0))
        t = torch.where(t < 2.0 * r, t, 2.0 * r)
        return torch.where(0.0 > t, torch.zeros_like(t), t)
    if meth == 2:
        t = torch.where(1.0 < 2.0 * r, torch.ones_like(r), 2.0 * r)
        u = torch.where(2.0 < r, torch.full_like(r, 2.0), r)
        t = torch.where(t > u, t, u)
        return torch.where(0.0 > t, torch.zeros_like(t), t)
    if meth == 3:
        return (r + torch.abs(r)) / (1.0 + torch.abs(r))
    if meth == 5:
        return r
    t = torch.where(1.0 < r, torch.ones_like(r), r)
    return torch.where(0.0 > t, torch.zeros_like(t), t)


def slice_fluxes(q1, a1, a2, a3, dtdx, trans, mthlim, order=2):
    """flux2 for one direction, all slices at once.

    q1: (3, n, L) cells along the last axis (L = len+4, padded);
    a2: aux of the slice, a1/a3: aux of the slices below/above (3 x (2, n, L)).
    Returns per-cell (qadd, fadd-difference input) pieces: qadd, fadd, gadd1,
    gadd2 over the padded cell index (only 1..len+... used by the caller)."""
    L = q1.shape[-1]
    # interfaces: right cell index k = 1..L-1 (left cell k-1)
    qL, qR = q1[..., :-1], q1[..., 1:]
    auxL, auxR = a2[..., :-1], a2[..., 1:]
    zi = auxR[0] * auxR[1]
    zim = auxL[0] * auxL[1]
    delta1 = qR[0] - qL[0]
    delta2 = qR[1] - qL[1]
    a1w = (-delta1 + zi * delta2) / (zim + zi)
    a2w = (delta1 + zim * delta2) / (zim + zi)
    zero = torch.zeros_like(a1w)
    W1 = torch.stack([-a1w * zim, a1w, zero])
    W2 = torch.stack([a2w * zi, a2w, zero])
    s1 = -auxL[1]
    s2 = auxR[1]
    amdq = torch.stack([s1 * W1[0], s1 * W1[1], s1 * W1[2]])
    apdq = torch.stack([s2 * W2[0], s2 * W2[1], s2 * W2[2]])
    # limiter on interfaces 1..len+1 (Fortran), i.e. interface index 1..L-3 here
    waves = [W1, W2]
    speeds = [s1, s2]
    lim = []
    for p in range(2):
        W = waves[p]
        meth = mthlim[p]
        if meth == 0:
            lim.append(W)
            continue
        wn = W[0] * W[0] + W[1] * W[1] + W[2] * W[2]
        inner = slice(1, W.shape[-1] - 1)
        Wc = W[..., inner]
        wnc = wn[..., inner]
        dotl = W[0][..., :-2] * Wc[0] + W[1][..., :-2] * Wc[1] + W[2][..., :-2] * Wc[2]
        dotr = Wc[0] * W[0][..., 2:] + Wc[1] * W[1][..., 2:] + Wc[2] * W[2][..., 2:]
        s = speeds[p][..., inner]
        dot = torch.where(s > 0.0, dotl, dotr)
        safe = torch.where(wnc == 0.0, torch.ones_like(wnc), wnc)
        phi = philim(safe, dot, meth)
        phi = torch.where(wnc == 0.0, torch.ones_like(phi), phi)
        Wl = torch.cat([W[..., :1], Wc * phi, W[..., -1:]], dim=-1)
        lim.append(Wl)
    dtdxave = 0.5 * (dtdx + dtdx)
    f = [torch.abs(sp) * (1.0 - torch.abs(sp) * dtdxave) for sp in speeds]
    cqxx = torch.stack([f[0] * lim[0][m] + f[1] * lim[1][m] for m in range(3)])
    if order == 1:
        cqxx = torch.zeros_like(cqxx)
    fadd = 0.5 * cqxx
    if trans == 2 and order == 2:
        A = amdq + cqxx
        P = apdq - cqxx
    else:
        A, P = amdq, apdq
    bm = [None, None]
    bp = [None, None]
    for ilr, asdq in ((1, A), (2, P)):
        sl = slice(0, -1) if ilr == 1 else slice(1, None)
        b1a, b2a, b3a = a1[..., sl], a2[..., sl], a3[..., sl]
        cm, cp = b1a[1], b3a[1]
        zm = b1a[0] * b1a[1]
        zz = b2a[0] * b2a[1]
        zp = b3a[0] * b3a[1]
        bb1 = (-asdq[0] + zz * asdq[2]) / (zm + zz)
        bb2 = (asdq[0] + zz * asdq[2]) / (zz + zp)
        z0 = torch.zeros_like(bb1)
        bm[ilr - 1] = torch.stack([cm * bb1 * zm, z0, -cm * bb1])
        bp[ilr - 1] = torch.stack([cp * bb2 * zp, z0, cp * bb2])
    return amdq, apdq, fadd, bm, bp


def step(qbc, auxbc, dt, dx, dy, trans=2, mthlim=(4, 4), bcl=(3, 3), bcu=(1, 1), abcl=(3, 3), abcu=(1, 1),
         order=2):
    """One unsplit step (step2.f90) on interior q; returns the new interior.

    qbc, auxbc: (3|2, mx+4, my+4) tensors whose interiors are used; ghost
    cells are refilled here from the interiors (differentiably)."""
    q = fill_bcs(qbc, bcl, bcu, True)
    aux = fill_bcs(auxbc, abcl, abcu, False)
    mx, my = q.shape[1] - 2 * G, q.shape[2] - 2 * G
    dtdx, dtdy = dt / dx, dt / dy
    hx, hy = 0.5 * dtdx, 0.5 * dtdy
    # ---- x slices j = 0..my+1 (Fortran) -> padded rows 1..my+2
    rows = slice(1, my + 3)
    qx = q[:, :, rows].permute(0, 2, 1)                   # (3, nrows, L) cells along x
    a1 = aux[:, :, 0:my + 2].permute(0, 2, 1)
    a2 = aux[:, :, 1:my + 3].permute(0, 2, 1)
    a3 = aux[:, :, 2:my + 4].permute(0, 2, 1)
    amdq, apdq, fadd, bm, bp = slice_fluxes(qx, a1, a2, a3, dtdx, trans, mthlim, order)
    # cell index c (padded 2..mx+1) uses interfaces c (left, index c-1 here) and c+1 (index c)
    cells = slice(2, mx + 2)
    il = slice(1, mx + 1)          # interface with right cell c  -> array index c-1
    ir = slice(2, mx + 2)          # interface with right cell c+1 -> array index c
    qadd = (0.0 - dtdx * apdq[..., il]) - dtdx * amdq[..., ir]
    dF = fadd[..., ir] - fadd[..., il]
    if trans > 0:
        g1 = (0.0 - hx * bm[0][..., ir]) - hx * bm[1][..., il]
        g2 = (0.0 - hx * bp[0][..., ir]) - hx * bp[1][..., il]
    # ---- y slices i = 0..mx+1 -> padded columns 1..mx+2
    cols = slice(1, mx + 3)
    qy = torch.stack([q[0], q[2], q[1]])[:, cols, :]      # swap u,v: normal component second
    b1 = aux[:, 0:mx + 2, :]
    b2 = aux[:, 1:mx + 3, :]
    b3 = aux[:, 2:mx + 4, :]
    amdqy, apdqy, faddy, bmy, bpy = slice_fluxes(qy, b1, b2, b3, dtdy, trans, mthlim, order)
    il2 = slice(1, my + 1)
    ir2 = slice(2, my + 2)
    qaddy = (0.0 - dtdy * apdqy[..., il2]) - dtdy * amdqy[..., ir2]
    dFy = faddy[..., ir2] - faddy[..., il2]
    if trans > 0:
        g1y = (0.0 - hy * bmy[0][..., ir2]) - hy * bmy[1][..., il2]
        g2y = (0.0 - hy * bpy[0][..., ir2]) - hy * bpy[1][..., il2]

    def unswap(t):
        return torch.stack([t[0], t[2], t[1]])

    qaddy, dFy = unswap(qaddy), unswap(dFy)
    if trans > 0:
        g1y, g2y = unswap(g1y), unswap(g2y)
    # ---- ordered accumulation per interior cell (step2.f90:139-145, 222-229)
    # x: rows r = padded 2..my+1 correspond to slice index r-1 in the x arrays
    v = q[:, cells, 2:my + 2].permute(0, 2, 1)            # (3, my, mx)
    if trans > 0:
        v = v + dtdy * g2[:, 0:my, :]                     # from slice j-1
    v = v + qadd[:, 1:my + 1, :] - dtdx * dF[:, 1:my + 1, :]
    if trans > 0:
        v = v - dtdy * (g2[:, 1:my + 1, :] - g1[:, 1:my + 1, :])
        v = v - dtdy * g1[:, 2:my + 2, :]                 # from slice j+1
    v = v.permute(0, 2, 1)                                # (3, mx, my)
    if trans > 0:
        v = v + dtdx * g2y[:, 0:mx, :]
        v = v + (qaddy[:, 1:mx + 1, :] - dtdy * dFy[:, 1:mx + 1, :] - dtdx * (g2y[:, 1:mx + 1, :] - g1y[:, 1:mx + 1, :]))
        v = v - dtdx * g1y[:, 2:mx + 2, :]
    else:
        v = v + (qaddy[:, 1:mx + 1, :] - dtdy * dFy[:, 1:mx + 1, :])
    return v


def padded(interior):
    t = torch.zeros((interior.shape[0], interior.shape[1] + 2 * G, interior.shape[2] + 2 * G), dtype=torch.float64)
    return _embed(t, interior)


def _embed(t, interior):
    mx, my = interior.shape[1], interior.shape[2]
    top = torch.zeros((t.shape[0], mx, G), dtype=t.dtype)
    col = torch.cat([top, interior, top], dim=2)
    side = torch.zeros((t.shape[0], G, my + 2 * G), dtype=t.dtype)
    return torch.cat([side, col, side], dim=1)


def run_shots(q0, aux, dt, dx, dy, src, rec, wavelet, **kw):
    """Multi-shot forward in plain torch: q0 (S,3,mx,my), aux (2,mx,my) ->
    traces (N,S,R).  After each step the wavelet sample wavelet[n, s] is added
    to the pressure of shot s's source cell src[s] = (i, j) (None: no source),
    then the pressure at every receiver rec[r] = (i, j) is recorded."""
    S = q0.shape[0]
    N = wavelet.shape[0]
    auxp = padded(aux)
    qs = [q0[s] for s in range(S)]
    ri = torch.tensor([c[0] for c in rec])
    rj = torch.tensor([c[1] for c in rec])
    out = []
    for n in range(N):
        row = []
        for s in range(S):
            qn = step(padded(qs[s]), auxp, dt, dx, dy, **kw)
            if src[s] is not None:
                i, j = src[s]
                qn = qn.index_put((torch.tensor([0]), torch.tensor([i]), torch.tensor([j])),
                                  wavelet[n, s].reshape(1), accumulate=True)
            qs[s] = qn
            row.append(qn[0][ri, rj])
        out.append(torch.stack(row))
    return torch.stack(out)
