"""Pure-PyTorch FP64 restatement of the discrete QUADESTH system (test infrastructure).

Differentiable with respect to the node coordinates and the material (nu, mu), so
autograd through it gives the reference gradient for the GPU adjoint.  Only tests use
it.  It covers 9-node quadrilateral meshes and small sizes: every (node, element) pair
and Gauss point is materialised as a tensor.

Follows the reference:
* Gauss points and weights of etaxja/extin8 (assembly_mod.f90:225-384): 6 x 6
  Gauss-Legendre points with the literal constants of assembly_mod.f90:6-19;
* singular elements by locin8/triloc8 (:386-616): the node's sub-triangles, each
  integrated with the collapsed 6 x 6 rule and weight N J (xi_i + 1) area / 4 w_i w_j;
* Kelvin kernels of funkelvin (:618-650) with the reference's index convention;
* the rigid-body diagonal H_ii = -sum_{j != i} H_ij (:100-123) and the column swap
  into A x = FI (:125-218), written with the summed H (exact when every element
  that prescribes a displacement at a node prescribes the same value);
* pinned DOFs as unit rows with zero right-hand side.
"""
from __future__ import annotations

import numpy as np
import torch

GI = [0.238619186083197, -0.238619186083197, 0.661209386466265,
      -0.661209386466265, 0.932469514203152, -0.932469514203152]
OME = [0.467913934572691, 0.467913934572691, 0.360761573048139,
       0.360761573048139, 0.171324492379170, 0.171324492379170]
PI = 3.14159265358979323846
Q1 = [-1.0, 0.0, 1.0, 1.0, 1.0, 0.0, -1.0, -1.0, 0.0]  # quad9 node parametric coordinates
Q2 = [-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0]


def shape9(g1, g2):
    """Quad9 shape functions and intrinsic derivatives at points (g1, g2): (..., 9)."""
    g1 = torch.as_tensor(g1, dtype=torch.float64)
    g2 = torch.as_tensor(g2, dtype=torch.float64)
    f = torch.stack([0.25 * g1 * g2 * (g1 - 1) * (g2 - 1), 0.5 * (1 - g1 * g1) * g2 * (g2 - 1),
                     0.25 * g1 * g2 * (g1 + 1) * (g2 - 1), 0.5 * g1 * (g1 + 1) * (1 - g2 * g2),
                     0.25 * g1 * g2 * (g1 + 1) * (g2 + 1), 0.5 * (1 - g1 * g1) * g2 * (g2 + 1),
                     0.25 * g1 * g2 * (g1 - 1) * (g2 + 1), 0.5 * g1 * (g1 - 1) * (1 - g2 * g2),
                     (1 - g1 * g1) * (1 - g2 * g2)], -1)
    d1 = torch.stack([0.25 * g2 * (g2 - 1) * (2 * g1 - 1), -g1 * g2 * (g2 - 1),
                      0.25 * g2 * (g2 - 1) * (2 * g1 + 1), 0.5 * (1 - g2 * g2) * (2 * g1 + 1),
                      0.25 * g2 * (g2 + 1) * (2 * g1 + 1), -g1 * g2 * (g2 + 1),
                      0.25 * g2 * (g2 + 1) * (2 * g1 - 1), 0.5 * (1 - g2 * g2) * (2 * g1 - 1),
                      -2 * g1 * (1 - g2 * g2)], -1)
    d2 = torch.stack([0.25 * g1 * (g1 - 1) * (2 * g2 - 1), 0.5 * (1 - g1 * g1) * (2 * g2 - 1),
                      0.25 * g1 * (g1 + 1) * (2 * g2 - 1), -g1 * g2 * (g1 + 1),
                      0.25 * g1 * (g1 + 1) * (2 * g2 + 1), 0.5 * (1 - g1 * g1) * (2 * g2 + 1),
                      0.25 * g1 * (g1 - 1) * (2 * g2 + 1), -g1 * g2 * (g1 - 1),
                      -2 * g2 * (1 - g1 * g1)], -1)
    return f, d1, d2


def _regular_rule():
    g1 = torch.tensor([GI[i] for i in range(6) for j in range(6)], dtype=torch.float64)
    g2 = torch.tensor([GI[j] for i in range(6) for j in range(6)], dtype=torch.float64)
    w = torch.tensor([OME[i] * OME[j] for i in range(6) for j in range(6)], dtype=torch.float64)
    return g1, g2, w


def _singular_rule(nodo: int):
    """(g1, g2, weight factor) of locin8's sub-triangle points for local node nodo
    (1-based), padded to 144 points with zero weight."""
    gii1 = Q1[:8] + Q1[:7]
    gii2 = Q2[:8] + Q2[:7]
    G1 = lambda p: gii1[p - 1]
    G2 = lambda p: gii2[p - 1]
    v0 = (Q1[nodo - 1], Q2[nodo - 1])
    tris = []
    if nodo in (1, 3, 5, 7):
        for k in (1, 2):
            m = 2 * k
            tris.append(((G1(nodo + m), G2(nodo + m)), (G1(nodo + m + 2), G2(nodo + m + 2)), 2.0))
    elif nodo in (2, 4, 6, 8):
        for k in (1, 2, 3):
            m = 2 * k - 1
            a = (G1(nodo + m), G2(nodo + m))
            b = (G1(nodo + m + 2), G2(nodo + m + 2))
            area = 0.5 * (a[0] * b[1] + v0[0] * a[1] + b[0] * v0[1] - a[0] * v0[1] - b[0] * a[1] - v0[0] * b[1])
            tris.append((a, b, area))
    else:
        for k in (1, 2, 3, 4):
            m = 2 * k - 1
            tris.append(((G1(m), G2(m)), (G1(m + 2), G2(m + 2)), 1.0))
    g1, g2, wf = [], [], []
    for a, b, area in tris:
        for i in range(6):
            for j in range(6):
                s1 = 0.5 * (GI[i] + 1.0)
                s2 = 0.5 * (GI[j] + 1.0)
                g1.append((1 - s1) * v0[0] + s1 * (1 - s2) * a[0] + s1 * s2 * b[0])
                g2.append((1 - s1) * v0[1] + s1 * (1 - s2) * a[1] + s1 * s2 * b[1])
                wf.append((GI[i] + 1.0) * area * 0.25 * OME[i] * OME[j])
    while len(g1) < 144:
        g1.append(0.0)
        g2.append(0.0)
        wf.append(0.0)
    return torch.tensor(g1, dtype=torch.float64), torch.tensor(g2, dtype=torch.float64), \
        torch.tensor(wf, dtype=torch.float64)


def _kelvin(rvec, n, c3, c4, c5, c6):
    """U*(jj, ii), T*(jj, ii) as (..., 3, 3) with [..., jj, ii] (funkelvin)."""
    r = torch.linalg.norm(rvec, dim=-1, keepdim=True)
    rd = rvec / r
    rdn = (rd * n).sum(-1, keepdim=True)
    eye = torch.eye(3, dtype=torch.float64)
    rr = rd.unsqueeze(-1) * rd.unsqueeze(-2)  # [..., jj, ii] = rd_jj rd_ii (symmetric)
    U = (c4 * eye + rr) * (c3 / r).unsqueeze(-1)
    nr = n.unsqueeze(-1) * rd.unsqueeze(-2)   # [..., jj, ii] = n_jj rd_ii
    T = (c5 / (r * r)).unsqueeze(-1) * (rdn.unsqueeze(-1) * (c6 * eye + 3.0 * rr) + c6 * (nr - nr.transpose(-1, -2)))
    return U, T


def _surface(Xe, f, d1, d2):
    """Points, Jacobians and unit normals: Xe (..., 9, 3), f/d1/d2 (..., q, 9)."""
    xg = torch.einsum("...qk,...kd->...qd", f, Xe)
    a1 = torch.einsum("...qk,...kd->...qd", d1, Xe)
    a2 = torch.einsum("...qk,...kd->...qd", d2, Xe)
    cr = torch.cross(a1, a2, dim=-1)
    J = torch.linalg.norm(cr, dim=-1)
    return xg, J, cr / J.unsqueeze(-1)


class System:
    """The discrete system of one quad9 mesh as differentiable torch tensors."""

    def __init__(self, mesh):
        assert (np.asarray(mesh.nconec) == 9).all(), "quad9 meshes only"
        self.mesh = mesh
        self.n, self.ne = mesh.n, mesh.ne
        self.kc = torch.as_tensor(np.asarray(mesh.kconec).T - 1, dtype=torch.long)  # (ne, 9)
        kode = np.asarray(mesh.kode).reshape(mesh.ne, 3)
        self.kode = kode
        # regular / singular pairs
        member = np.zeros((mesh.n, mesh.ne), dtype=np.int64)  # local node + 1 of node i in e
        for e in range(mesh.ne):
            for k in range(9):
                member[mesh.kconec[k, e] - 1, e] = k + 1
        self.member = torch.as_tensor(member)
        si, se = np.nonzero(member)
        self.sing_i = torch.as_tensor(si)
        self.sing_e = torch.as_tensor(se)
        self.sing_nodo = torch.as_tensor(member[si, se])
        rules = [_singular_rule(nd) for nd in range(1, 10)]
        self.srule = [torch.stack([r[c] for r in rules]) for c in range(3)]  # (9, 144) each
        self.greg = _regular_rule()
        # column-swap bookkeeping (u known per dof: first element in adjacency order)
        N = 3 * mesh.n
        uk = np.zeros(N, dtype=bool)
        vp = np.zeros(N)
        order = [[] for _ in range(mesh.n)]
        for e in range(mesh.ne):
            for k in range(9):
                order[mesh.kconec[k, e] - 1].append((e, k))
        for i in range(mesh.n):
            for ld in range(3):
                for e, k in order[i][:8]:
                    if kode[e, ld] == 0:
                        uk[3 * i + ld] = True
                        vp[3 * i + ld] = mesh.bc[3 * k + ld, e]
                        break
        self.uk = torch.as_tensor(uk)
        self.vp = torch.as_tensor(vp)
        self.pins = torch.as_tensor(np.asarray(mesh.pins, dtype=np.int64))

    def hg(self, X, mu, nu):
        """H (3n x 3n, rigid-body diagonal included) and G (3n x 27 ne)."""
        n, ne = self.n, self.ne
        c3 = 1.0 / (16.0 * PI * (1.0 - nu) * mu)
        c4 = 3.0 - 4.0 * nu
        c5 = -1.0 / (8.0 * PI * (1.0 - nu))
        c6 = 1.0 - 2.0 * nu
        Xe = X[self.kc]  # (ne, 9, 3)
        g1, g2, w = self.greg
        f, d1, d2 = shape9(g1, g2)  # (36, 9)
        xg, J, nrm = _surface(Xe, f.expand(ne, 36, 9), d1.expand(ne, 36, 9), d2.expand(ne, 36, 9))
        p12 = f.unsqueeze(0) * (J * w).unsqueeze(-1)  # (ne, 36, 9)
        rvec = xg.unsqueeze(0) - X[:, None, None, :]  # (n, ne, 36, 3)
        U, T = _kelvin(rvec, nrm.unsqueeze(0), c3, c4, c5, c6)  # (n, ne, 36, 3, 3)
        g = torch.einsum("ieqab,eqk->iekab", U, p12)  # [i, e, k, jj, ii]
        h = torch.einsum("ieqab,eqk->iekab", T, p12)
        reg = (self.member == 0).to(torch.float64)[:, :, None, None, None]
        g = g * reg
        h = h * reg
        # singular pairs
        si, se, nodo = self.sing_i, self.sing_e, self.sing_nodo
        sg1, sg2, swf = (r[nodo - 1] for r in self.srule)  # (P, 144)
        fs, ds1, ds2 = shape9(sg1, sg2)  # (P, 144, 9)
        xs, Js, ns = _surface(X[self.kc[se]], fs, ds1, ds2)
        ps = fs * (Js * swf).unsqueeze(-1)
        rs = xs - X[si].unsqueeze(1)
        rs = torch.where(swf.unsqueeze(-1) > 0, rs, torch.ones_like(rs))  # padded points
        Us, Ts = _kelvin(rs, ns, c3, c4, c5, c6)
        gs = torch.einsum("pqab,pqk->pkab", Us, ps)
        hs = torch.einsum("pqab,pqk->pkab", Ts, ps)
        keep = (torch.arange(9)[None, :] != (nodo - 1)[:, None]).to(torch.float64)[:, :, None, None]
        hs = hs * keep  # the entry at the singular node is replaced by the rigid-body sum
        g = g.index_put((si, se), gs, accumulate=True)
        h = h.index_put((si, se), hs, accumulate=True)
        # G: (3n, 27 ne), G[3i + jj, 27e + 3k + ii]
        G = g.permute(0, 3, 1, 2, 4).reshape(3 * n, 27 * ne)
        # H: scatter h[i, e, k, jj, ii] into column 3 kc[e, k] + ii
        cols = (3 * self.kc[:, :, None] + torch.arange(3)[None, None, :]).reshape(-1)  # (ne*27)
        hh = h.permute(0, 3, 1, 2, 4).reshape(3 * n, 27 * ne)
        H = torch.zeros(3 * n, 3 * n, dtype=torch.float64).index_add(1, cols, hh)
        # rigid-body diagonal: H_ii = -sum_{j != i} H_ij
        Hb = H.reshape(n, 3, n, 3)
        off = Hb.sum(2)  # (n, 3, 3): row block sums (the diagonal blocks are zero so far)
        eye_n = torch.eye(n, dtype=torch.float64)
        H = (Hb - eye_n[:, None, :, None] * off[:, :, None, :]).reshape(3 * n, 3 * n)
        return H, G

    def system(self, X, mu, nu):
        """A and FI (assembly_mod.f90:125-218, pins applied)."""
        H, G = self.hg(X, mu, nu)
        n, ne, N = self.n, self.ne, 3 * self.n
        m = self.mesh
        A = torch.where(self.uk[None, :], torch.zeros_like(H), H)
        FI = -(H[:, self.uk] * self.vp[self.uk]).sum(1)
        for e in range(ne):
            for k in range(9):
                ik = int(m.kconec[k, e]) - 1
                for ld in range(3):
                    gc = G[:, 27 * e + 3 * k + ld]
                    if self.kode[e, ld] == 0:
                        A = A.index_add(1, torch.tensor([3 * ik + ld]), (-mu * gc)[:, None])
                    else:
                        b = float(m.bc[3 * k + ld, e])
                        if b != 0.0:
                            FI = FI + gc * b
        if len(self.pins):
            rows = self.pins
            A = A.index_fill(0, rows, 0.0)
            A = A.index_put((rows, rows), torch.ones(len(rows), dtype=torch.float64))
            FI = FI.index_fill(0, rows, 0.0)
        return A, FI

    def reorganize(self, x, mu):
        """u (3n) and t (27 ne) of the solution (io_mod.f90:148-183)."""
        m = self.mesh
        u = torch.where(self.uk, self.vp, x)
        cols = []
        for e in range(self.ne):
            for k in range(9):
                ik = int(m.kconec[k, e]) - 1
                for ld in range(3):
                    cols.append(mu * x[3 * ik + ld] if self.kode[e, ld] == 0
                                else torch.tensor(float(m.bc[3 * k + ld, e]), dtype=torch.float64))
        return u, torch.stack(cols)

    def compliance(self, X, u, t, elements):
        """J = sum over `elements` of the integral of t . u (6 x 6 Gauss points)."""
        g1, g2, w = self.greg
        f, d1, d2 = shape9(g1, g2)
        el = torch.as_tensor(np.asarray(elements, dtype=np.int64))
        Xe = X[self.kc[el]]
        _, J, _ = _surface(Xe, f.expand(len(el), 36, 9), d1.expand(len(el), 36, 9), d2.expand(len(el), 36, 9))
        ue = u.reshape(self.n, 3)[self.kc[el]]          # (E, 9, 3)
        te = t.reshape(self.ne, 9, 3)[el]               # (E, 9, 3)
        uq = torch.einsum("qk,ekd->eqd", f, ue)
        tq = torch.einsum("qk,ekd->eqd", f, te)
        return ((uq * tq).sum(-1) * J * w).sum()

    def objective(self, X, mu, nu, elements):
        """Solve the system and return (J, x)."""
        A, FI = self.system(X, mu, nu)
        x = torch.linalg.solve(A, FI)
        u, t = self.reorganize(x, mu)
        return self.compliance(X, u, t, elements), x
