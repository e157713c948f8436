"""Row-partitioned CPR-GMRES: one system spread over several GPUs.

The reference distributes a system as contiguous row blocks whose sizes are
multiples of the block size (IO/cpp_read.hpp:454-459, split_rows), keeps global
column indices, and before every product sends each rank's whole x block to the
ranks that reference it, into a global-length buffer (core/alg.hpp:81-144,
MPI_spmv); dot products end in an all-reduce (core/alg.hpp:309-327).  Here:

- the same bs-aligned row blocks and global column indices;
- a halo plan per operator (`Halo`): for every other rank, the ghost columns this
  rank's rows read that it owns (received) and the columns of this rank that it
  reads (sent), exchanged once at setup; before a product only those entries
  move (point-to-point over torch.distributed: NCCL between GPUs, gloo on CPU)
  into a global-length buffer, as in the reference;
- right GMRES(m) with the single-GPU path's Arnoldi step (CGS2 with the second
  projection from the Gram matrix): the block of dots h = V^T w and the Gram row
  V^T v_j of an Arnoldi step is ONE all-reduce; ||w''|| a second;
- CPR seq 3 applied with row slices of its operators (decoupled A, global FSAI
  FL and FU^T, pressure FSAI FL and FU^T): each operator reads its ghosts through
  its own halo plan (FL rows only lower ones, FU^T rows only upper ones).

Setup is replicated: every rank runs the whole CPR setup (decoupling, A_pp, both
FSAI setups) on its own device and keeps its row slices.  The decoupling is
cell-local and the FSAI rows are independent, so a row-partitioned setup would
produce the same rows; replicating it costs setup time and memory but keeps each
rank's preconditioner rows bit-identical to the single-GPU ones, so the
distributed solve needs the single-GPU iteration count (up to the order of the
reduced dot products).  The in-house FSAI of the reference is itself single-rank
(README.md:10-12).

The local products go through a product backend: `LibraryProducts` (the
library's CSR SpMV on device row slices, the product path) or any object with the
same two methods (the CPU tests use scipy).  Vectors are torch tensors on the
backend's device; the GMRES recurrences run in float64.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def split_rows(n: int, world: int, bs: int = 1) -> list[int]:
    """Row offsets of the `world` blocks: every block but the last holds
    floor(n / world) rows rounded down to a multiple of bs; the last takes the rest
    (IO/cpp_read.hpp:454-459)."""
    if world < 1 or n < 0 or bs < 1:
        raise ValueError("bad split")
    nloc = n // world
    if nloc % bs:
        nloc = (nloc // bs) * bs
    return [k * nloc for k in range(world)] + [n]


def _dist():
    import torch.distributed as dist
    return dist if (dist.is_available() and dist.is_initialized()) else None


class Halo:
    """Ghost entries of a row slice: which global columns outside this rank's block
    its rows read, grouped by owner, and which of this rank's entries the other
    ranks read.  Built collectively (every rank calls it with its own columns)."""

    def __init__(self, cols: np.ndarray, displs: list[int], rank: int, world: int, device):
        import torch
        self.rank, self.world = rank, world
        lo, hi = displs[rank], displs[rank + 1]
        cols = np.unique(np.asarray(cols, np.int64))
        ghost = cols[(cols < lo) | (cols >= hi)]
        owner = np.searchsorted(np.asarray(displs[1:], np.int64), ghost, side="right")
        self.recv = {q: ghost[owner == q] for q in range(world) if q != rank and np.any(owner == q)}
        dist = _dist()
        if world > 1:
            if dist is None:
                raise RuntimeError("a row-partitioned solve over several ranks needs torch.distributed")
            wanted = [None] * world
            dist.all_gather_object(wanted, {q: v.tolist() for q, v in self.recv.items()})
            self.send = {q: np.asarray(wanted[q][rank], np.int64) for q in range(world)
                         if q != rank and rank in wanted[q]}
        else:
            self.send = {}
        self.device = device
        self.recv_t = {q: torch.as_tensor(v, dtype=torch.long, device=device) for q, v in self.recv.items()}
        self.send_t = {q: torch.as_tensor(v, dtype=torch.long, device=device) for q, v in self.send.items()}

    @property
    def ghosts(self) -> int:
        return sum(len(v) for v in self.recv.values())

    def exchange(self, xg):
        """Fill the ghost entries of the global-length buffer `xg` (this rank's block
        already current) from their owners; send this rank's entries to the ranks
        that read them.  Every receive is posted before any send."""
        if not self.recv and not self.send:
            return
        import torch
        dist = _dist()
        bufs, reqs = {}, []
        for q in sorted(self.recv_t):
            bufs[q] = torch.empty(len(self.recv_t[q]), dtype=xg.dtype, device=xg.device)
            reqs.append(dist.irecv(bufs[q], src=q))
        out = []
        for q in sorted(self.send_t):
            t = xg.index_select(0, self.send_t[q])
            out.append(t)
            reqs.append(dist.isend(t, dst=q))
        for r in reqs:
            r.wait()
        for q, b in bufs.items():
            xg.index_copy_(0, self.recv_t[q], b)


@dataclass
class RowSlice:
    """Rows [r0, r1) of a global CSR matrix with global column indices."""
    r0: int
    r1: int
    ncols: int
    r: np.ndarray
    c: np.ndarray
    v: np.ndarray

    @classmethod
    def cut(cls, r, c, v, r0, r1, ncols):
        a, e = int(r[r0]), int(r[r1])
        return cls(r0, r1, ncols, (np.asarray(r[r0:r1 + 1], np.int64) - a).astype(np.int32),
                   np.ascontiguousarray(c[a:e], np.int32), np.ascontiguousarray(v[a:e], np.float64))

    @property
    def rows(self) -> int:
        return self.r1 - self.r0


class LibraryProducts:
    """Local products through the library's CSR SpMV on device row slices (deco_spmv:
    full rows, or the restricted row-0-of-every-cell form)."""

    def __init__(self, ctx=None):
        import torch
        from . import default_context
        self.ctx = ctx or default_context()
        self.device = torch.device("cuda", self.ctx.device)

    def prepare(self, sl: RowSlice):
        from . import CSR
        return CSR(sl.rows, sl.ncols, sl.r, sl.c, sl.v, self.ctx)

    def apply(self, M, xg, bs: int = 1):
        return M.apply(xg, bs=bs)


class DistCPR:
    """CPR seq 3 (precond/CPR.hpp:235-274) applied to this rank's rows, from row
    slices of the operators of a CPR setup on the whole system."""

    def __init__(self, ops, displs, rank, world, bs, pid, A, FL, FUt, FLp, FUtp):
        import torch
        self.ops, self.bs, self.p = ops, bs, pid
        self.rank, self.world = rank, world
        self.displs = displs
        self.cdispls = [d // bs for d in displs]
        dev = ops.device
        self.n, self.nc = displs[-1], self.cdispls[-1]
        self.r0, self.r1 = displs[rank], displs[rank + 1]
        self.c0, self.c1 = self.cdispls[rank], self.cdispls[rank + 1]
        self.A, self.FL, self.FUt = (ops.prepare(m) for m in (A, FL, FUt))
        self.FLp, self.FUtp = (ops.prepare(m) for m in (FLp, FUtp))
        self.hA = Halo(A.c, displs, rank, world, dev)
        self.hFL = Halo(FL.c, displs, rank, world, dev)
        self.hFUt = Halo(FUt.c, displs, rank, world, dev)
        self.hFLp = Halo(FLp.c, self.cdispls, rank, world, dev)
        self.hFUtp = Halo(FUtp.c, self.cdispls, rank, world, dev)
        f64 = dict(dtype=torch.float64, device=dev)
        self.gx = torch.zeros(self.n, **f64)    # global-length buffers (own block + ghosts)
        self.gt = torch.zeros(self.n, **f64)
        self.gp = torch.zeros(self.nc, **f64)
        self.gq = torch.zeros(self.nc, **f64)

    def product(self, M, halo, g, lo, hi, x, bs=1):
        g[lo:hi] = x
        halo.exchange(g)
        return self.ops.apply(M, g, bs)

    def glo(self, r):  # FU^T (FL r) of FSAI::precond (precond/FSAI/FSAI.hpp:40-47)
        t = self.product(self.FL, self.hFL, self.gt, self.r0, self.r1, r)
        return self.product(self.FUt, self.hFUt, self.gt, self.r0, self.r1, t)

    def apply(self, r):
        bs, p = self.bs, self.p
        x = self.glo(r)
        ax0 = self.product(self.A, self.hA, self.gx, self.r0, self.r1, x, bs)   # row 0 of every cell
        rts = r[p::bs] - ax0
        tl = self.product(self.FLp, self.hFLp, self.gp, self.c0, self.c1, rts)
        xp = self.product(self.FUtp, self.hFUtp, self.gq, self.c0, self.c1, tl)
        x[p::bs] += xp
        rt = r - self.product(self.A, self.hA, self.gx, self.r0, self.r1, x)
        x += self.glo(rt)
        return x

    def matvec(self, x):
        return self.product(self.A, self.hA, self.gx, self.r0, self.r1, x)


def _allreduce(t):
    dist = _dist()
    if dist is not None and dist.get_world_size() > 1:
        dist.all_reduce(t)
    return t


def _givens(x, y, eps=2.220446049250312e-16):  # solver/rgmres.tpp:141-153
    if abs(y) < eps:
        return 1.0, 0.0
    if abs(y) > abs(x):
        nu = x / y
        s = 1.0 / np.sqrt(1.0 + nu * nu)
        return nu * s, s
    nu = y / x
    c = 1.0 / np.sqrt(1.0 + nu * nu)
    return c, nu * c


def _rot(c, s, dx, dy):  # solver/rgmres.tpp:155-160
    return c * dx + s * dy, -s * dx + c * dy


def rgmres(P: DistCPR, b, restart=50, reltol=1e-8, itmax=3000):
    """Right-preconditioned GMRES(m) on this rank's rows (solver/rgmres.tpp:8-139):
    the reference's inner check |g_j| < tol ||b|| before every step and outer
    check on the true residual after every restart.  Arnoldi step: h = V^T w and
    the Gram row V^T v_j in one all-reduce, c = h + (h - G h) (CGS2 with the second
    projection from the Gram matrix), w'' = w - V c, ||w''|| in a second all-reduce.
    Returns (x on this rank's rows, iterations, ||b - A x|| / ||b||, flag)."""
    import torch
    m = int(restart)
    nl = b.numel()
    dev, f64 = b.device, torch.float64
    V = torch.zeros(m + 1, nl, dtype=f64, device=dev)
    H = np.zeros((m + 1, m))
    G = np.zeros((m + 1, m + 1))
    x = torch.zeros(nl, dtype=f64, device=dev)
    bnorm = float(_allreduce(torch.dot(b, b).reshape(1))[0]) ** 0.5
    abstol = reltol * bnorm
    r = b.clone()
    it, flag, rnorm = 0, 1, bnorm
    while it < itmax:
        g = np.zeros(m + 1)
        cs, sn = np.zeros(m), np.zeros(m)
        g[0] = float(_allreduce(torch.dot(r, r).reshape(1))[0]) ** 0.5
        V[0] = r / g[0]
        j = 0
        while j < m and it < itmax:
            rnorm = abs(g[j])
            if rnorm < abstol:
                flag = 0
                break
            w = P.matvec(P.apply(V[j].clone()))
            loc = torch.cat([V[:j + 1] @ w, V[:j + 1] @ V[j]])
            red = _allreduce(loc).cpu().numpy()
            h, gr = red[:j + 1], red[j + 1:]
            G[:j + 1, j] = gr
            G[j, :j + 1] = gr
            c = h + (h - G[:j + 1, :j + 1] @ h)
            w = w - V[:j + 1].T @ torch.as_tensor(c, dtype=f64, device=dev)
            beta = float(_allreduce(torch.dot(w, w).reshape(1))[0]) ** 0.5
            H[:j + 1, j] = c
            H[j + 1, j] = beta
            V[j + 1] = w / beta if beta != 0.0 else w
            for i in range(j):
                H[i, j], H[i + 1, j] = _rot(cs[i], sn[i], H[i, j], H[i + 1, j])
            cs[j], sn[j] = _givens(H[j, j], H[j + 1, j])
            H[j, j], H[j + 1, j] = _rot(cs[j], sn[j], H[j, j], H[j + 1, j])
            g[j], g[j + 1] = _rot(cs[j], sn[j], g[j], g[j + 1])
            j += 1
            it += 1
        y = g.copy()
        for i in range(j - 1, -1, -1):  # rgmres.tpp:95-104
            if H[i, i] == 0.0:
                raise ArithmeticError("Error in rgmres: Zero diagonal element in upper triangular matrix.")
            y[i] /= H[i, i]
            y[:i] -= H[:i, i] * y[i]
        k = max(j, 1)
        z = V[:k].T @ torch.as_tensor(y[:k], dtype=f64, device=dev)
        x += P.apply(z)
        r = b - P.matvec(x)
        rnorm = float(_allreduce(torch.dot(r, r).reshape(1))[0]) ** 0.5
        if rnorm < abstol:
            flag = 0
            break
    return x, it, rnorm / bnorm, flag


def slices_from_cpr(P, A, bs, displs, rank):
    """This rank's row slices of the operators of a CPR setup on the whole system
    (`deco_b200.CPR` after it decoupled `A`): decoupled A, the global FSAI's FL and
    FU^T, and the pressure FSAI's FL and FU^T (on the cell index space)."""
    n = displs[-1]
    nc = n // bs
    r0, r1 = displs[rank], displs[rank + 1]
    c0, c1 = r0 // bs, r1 // bs
    Ar, Ac, Av = A.download()
    (Lr, Lc, Lv), (Ur, Uc, Uv) = P.fsai(0).factors()
    (lr, lc, lv), (ur, uc, uv) = P.fsai(1).factors()
    return (RowSlice.cut(Ar, Ac, Av, r0, r1, n), RowSlice.cut(Lr, Lc, Lv, r0, r1, n),
            RowSlice.cut(Ur, Uc, Uv, r0, r1, n), RowSlice.cut(lr, lc, lv, c0, c1, nc),
            RowSlice.cut(ur, uc, uv, c0, c1, nc))


def solve(prec: dict, sysm, sol: dict, rank: int = 0, world: int = 1, ctx=None):
    """Row-partitioned CPR(FSAI, FSAI) seq 3 + rgmres of a system every rank holds on
    the host (`sysm` with r, c, v, b): the CPR setup runs on this rank's device
    for the whole system, the solve on this rank's rows.  Returns
    (x on this rank's rows, iterations, relative residual on the decoupled system,
    flag, row offsets).  Under torchrun each rank passes its RANK and WORLD_SIZE,
    with a process group initialised (NCCL for GPUs)."""
    import torch
    from . import CPR, CSR
    ops = LibraryProducts(ctx)
    bs = int(prec["block_size"])
    pid = int(prec.get("pressure_id", 0))
    if str(prec.get("seq", "3")) != "3" or prec["prec_glo"]["type"] != "FSAI" or prec["prec_loc"]["type"] != "FSAI":
        raise ValueError("the row-partitioned solve runs CPR seq 3 with FSAI stages")
    n = len(sysm.r) - 1
    displs = split_rows(n, world, bs)
    A = CSR(n, n, sysm.r, sysm.c, sysm.v, ops.ctx)
    bg = torch.from_numpy(np.ascontiguousarray(sysm.b, np.float64)).to(ops.device)
    P = CPR(prec, A, bg)
    sl = slices_from_cpr(P, A, bs, displs, rank)
    D = DistCPR(ops, displs, rank, world, bs, pid, *sl)
    bl = bg[displs[rank]:displs[rank + 1]].clone()
    del P, A
    x, it, res, flag = rgmres(D, bl, int(sol["restart"]), float(sol["reltol"]), int(sol["itmax"]))
    return x, it, res, flag, displs
