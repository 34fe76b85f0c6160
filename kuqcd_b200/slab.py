"""Domain decomposition along t: one slab of the global lattice per rank (one GPU per rank), halo exchange through
a transport, and the reference's multishift CG (inverter_cgm.cpp:17-87) over the slabs with its reductions summed
across ranks (spinor_field.cpp:207-215, 235-243).

The kernels are in libkuqcd_b200.so (kq_slab.cu): face packing into the sender's buffers and a dslash that reads
the received ghost buffers in place.  Transports move the faces:

    TorchTransport   one rank per process over torch.distributed: NCCL for device buffers (NVLink), gloo for host
                     buffers.  Two phases per exchange (faces going up in t, then down), so that with two ranks the
                     point-to-point messages between the same pair are matched in order.
    LocalTransport   every rank in this process: the ghost of a rank IS its neighbour's face buffer (no copy).
                     Used to run a decomposed solve on one GPU, where ranks cannot run concurrently.

Code written against a list of local slabs runs unchanged under both (SPMD over `slabs`).

    slabs = [Slab(global_dims, r, R) for r in range(R)]              # or [Slab(global_dims, rank, world)]
    for s in slabs: s.load_links(slab_of_links(fat, global_dims, s.rank, R), slab_of_links(lng, ...))
    exchange_link_ghosts(slabs, transport)
    xs, iters = cgm(slabs, transport, [b_r ...], shifts_ref, tol, max_iter)
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import lib as L


def _p(t):
    return L._ptr(t)


# parts of a slab's output sites (kq_slab_dslash_part)
PART_ALL, PART_INTERIOR, PART_BOUNDARY = 0, 1, 2


# ---------------------------------------------------------------------------------------------------- host slicing
def slab_of_links(record: np.ndarray, global_dims, rank: int, nranks: int) -> np.ndarray:
    """Local NORMAL_ORDER link record (even sites then odd sites, 72 values per site) of one rank's slab."""
    nx, ny, nz, nt = global_dims
    lt, S = nt // nranks, nx * ny * nz // 2
    vh = nx * ny * nz * nt // 2
    rec = record.reshape(2, vh, 72)
    return np.ascontiguousarray(rec[:, rank * lt * S:(rank + 1) * lt * S]).reshape(-1)


def slab_of_spinor(record: np.ndarray, global_dims, rank: int, nranks: int) -> np.ndarray:
    """Local record (Vh_local * 6 values) of one parity field."""
    nx, ny, nz, nt = global_dims
    lt, S = nt // nranks, nx * ny * nz // 2
    return np.ascontiguousarray(record.reshape(-1, 6)[rank * lt * S:(rank + 1) * lt * S]).reshape(-1)


def join_spinor(parts) -> np.ndarray:
    """Inverse of slab_of_spinor over all ranks (t is the slowest index of the checkerboard order)."""
    return np.concatenate([np.asarray(p).reshape(-1) for p in parts])


# ---------------------------------------------------------------------------------------------------- transports
class LocalTransport:
    """All ranks in this process: ghosts are the neighbours' face buffers; reductions are plain sums."""

    def exchange(self, faces):
        R = len(faces)
        return [(faces[(r - 1) % R][1], faces[(r + 1) % R][0]) for r in range(R)]

    def exchange_start(self, faces):
        return faces

    def exchange_wait(self, handle):
        return self.exchange(handle)

    def allreduce(self, values):
        tot = np.sum(np.asarray(values, dtype=np.float64), axis=0)
        return [tot.copy() for _ in values]

    def allreduce_inplace(self, tensors):
        """Every rank's device tensor becomes the sum over ranks, in stream order (no host synchronisation)."""
        tot = torch.stack([t.to(tensors[0].device) for t in tensors]).sum(0)
        for t in tensors:
            t.copy_(tot)


class TorchTransport:
    """One rank per process over torch.distributed (the process group must exist)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def _peer(self, d):
        r = (self.rank + d) % self.world
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def exchange(self, faces):
        return self.exchange_wait(self.exchange_start(faces))

    def exchange_start(self, faces):
        """Posts the first phase (faces going up in t) and returns at once: work that reads no ghost (the interior
        dslash) can run while it is in flight."""
        (lo, hi), = faces
        if self.world == 1:
            return (lo, hi, None, None, None)
        d = self.dist
        ghost_lo, ghost_hi = torch.empty_like(hi), torch.empty_like(lo)
        # up in t: my top face becomes the lower ghost of rank + 1
        ops = [d.P2POp(d.isend, hi, self._peer(1), self.group), d.P2POp(d.irecv, ghost_lo, self._peer(-1), self.group)]
        return (lo, hi, ghost_lo, ghost_hi, d.batch_isend_irecv(ops))

    def exchange_wait(self, handle):
        lo, hi, ghost_lo, ghost_hi, works = handle
        if works is None:
            return [(hi, lo)]
        d = self.dist
        for w in works:
            w.wait()
        # down in t: my bottom face becomes the upper ghost of rank - 1 (a second phase, so that two ranks, whose
        # neighbours are the same peer, match their messages in order)
        ops = [d.P2POp(d.isend, lo, self._peer(-1), self.group), d.P2POp(d.irecv, ghost_hi, self._peer(1), self.group)]
        for w in d.batch_isend_irecv(ops):
            w.wait()
        # on CUDA, wait() orders torch's current stream after the transfers, and the slab kernels run on that stream
        return [(ghost_lo, ghost_hi)]

    def allreduce(self, values):
        (v,) = values
        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor(np.asarray(v, dtype=np.float64), device=dev)
        self.dist.all_reduce(t, group=self.group)
        return [t.cpu().numpy()]

    def allreduce_inplace(self, tensors):
        """This rank's tensor becomes the sum over ranks: NCCL on the device in stream order (no host
        synchronisation); gloo through the host."""
        (t,) = tensors
        if self.dist.get_backend(self.group) == "nccl":
            self.dist.all_reduce(t, group=self.group)
        else:
            h = t.cpu()
            self.dist.all_reduce(h, group=self.group)
            t.copy_(h)


# ---------------------------------------------------------------------------------------------------- one slab
class Slab:
    """One rank's slab: a context of the local lattice (nx, ny, nz, nt / nranks) marked as slab `rank`."""

    def __init__(self, global_dims, rank: int, nranks: int, device: int = 0):
        nx, ny, nz, nt = global_dims
        if nt % nranks:
            raise ValueError("nt must be a multiple of the number of ranks")
        self.global_dims = tuple(global_dims)
        self.rank, self.nranks = rank, nranks
        self.dims = (nx, ny, nz, nt // nranks)
        self.device = device
        self.ctx = L.Context(self.dims, device)
        self.ctx._chk(L.library().kq_slab_set(self.ctx._h, rank, nranks), "kq_slab_set")
        self._faces = {}

    def stream(self):
        """torch's current stream on the slab's device: every slab operation, the transport's NCCL calls and the
        caller's tensor operations are ordered on it, so no step needs a host synchronisation"""
        return L._torch_stream(self.device)

    def field(self, prec=L.KUQCD_DOUBLE):
        return torch.zeros(self.ctx.spinor_bytes(prec), dtype=torch.uint8, device=f"cuda:{self.device}")

    def load_links(self, fat_local, lng_local):
        self.ctx.load_links(L.KUQCD_FAT_LINK, fat_local)
        self.ctx.load_links(L.KUQCD_LONG_LINK, lng_local)

    def link_face(self):
        n = L.library().kq_slab_link_face_bytes(self.ctx._h)
        f = torch.empty(n, dtype=torch.uint8, device=f"cuda:{self.device}")
        self.ctx._chk(L.library().kq_slab_pack_link_face(self.ctx._h, _p(f)), "kq_slab_pack_link_face")
        return f

    def set_link_ghosts(self, face):
        self.ctx._chk(L.library().kq_slab_set_link_ghosts(self.ctx._h, _p(face)), "kq_slab_set_link_ghosts")

    def pack(self, prec, src):
        """(face_lo, face_hi) of src; the buffers are reused by the next pack of the same precision."""
        if prec not in self._faces:
            n = L.library().kq_slab_face_bytes(self.ctx._h, prec)
            self._faces[prec] = tuple(torch.empty(n, dtype=torch.uint8, device=f"cuda:{self.device}")
                                      for _ in range(2))
        lo, hi = self._faces[prec]
        self.ctx._chk(L.library().kq_slab_pack_faces(self.ctx._h, prec, _p(src), _p(lo), _p(hi), self.stream()),
                      "kq_slab_pack_faces")
        return lo, hi

    def dslash(self, prec, src, ghost_lo, ghost_hi, dst, dst_parity, pvec=None, sigma=0.0, part=PART_ALL):
        self.ctx._chk(L.library().kq_slab_dslash_part(self.ctx._h, prec, _p(src), _p(ghost_lo), _p(ghost_hi),
                                                      _p(dst), dst_parity, _p(pvec), float(sigma), part,
                                                      self.stream()),
                      "kq_slab_dslash_part")

    def dot_device(self, x, y, out):
        """local <x, y> into out (a one-element float64 device tensor), without a host round trip"""
        self.ctx._chk(L.library().kq_field_dot_device(self.ctx._h, _p(x), _p(y), _p(out), self.stream()),
                      "kq_field_dot_device")

    def axpby(self, a, x, b, y):
        self.ctx._chk(L.library().kq_field_axpby(self.ctx._h, float(a), _p(x), float(b), _p(y), self.stream()),
                      "kq_field_axpby")

    # device-driven multishift CG (kq_slab_cgm_*): the state is a float64 device tensor whose first two elements are
    # the sums the transport all-reduces in place
    def cgm_state(self):
        n = L.library().kq_slab_cgm_state_bytes()
        return torch.zeros(n // 8, dtype=torch.float64, device=f"cuda:{self.device}")

    def cgm_init(self, state, shifts_ref, tol, max_iter):
        sh = np.ascontiguousarray(shifts_ref, dtype=np.float64)
        self.ctx._chk(L.library().kq_slab_cgm_init(self.ctx._h, _p(state), len(sh),
                                                   sh.ctypes.data_as(C.POINTER(C.c_double)), float(tol),
                                                   int(max_iter), self.stream()), "kq_slab_cgm_init")

    def cgm_step(self, state, step):
        self.ctx._chk(L.library().kq_slab_cgm_step(self.ctx._h, _p(state), step, self.stream()), "kq_slab_cgm_step")

    def cgm_residual(self, state, s, r):
        self.ctx._chk(L.library().kq_slab_cgm_residual(self.ctx._h, _p(state), _p(s), _p(r), self.stream()),
                      "kq_slab_cgm_residual")

    def cgm_update(self, state, r, p_block, x_block):
        vb = self.ctx.spinor_bytes(L.KUQCD_DOUBLE)
        self.ctx._chk(L.library().kq_slab_cgm_update(self.ctx._h, _p(state), _p(r), _p(p_block), _p(x_block), vb,
                                                     self.stream()), "kq_slab_cgm_update")

    def cgm_poll(self, state, with_rr=False):
        """(iterations, stopped[, |r|^2]) of the state; waits for the stream"""
        it, done, rr = C.c_int(), C.c_int(), C.c_double()
        self.ctx._chk(L.library().kq_slab_cgm_poll(self.ctx._h, _p(state), C.byref(it), C.byref(done),
                                                   C.byref(rr), self.stream()), "kq_slab_cgm_poll")
        return (it.value, bool(done.value), rr.value) if with_rr else (it.value, bool(done.value))

    def dot(self, x, y) -> float:
        out = C.c_double()
        L._torch_wait(self.device)  # kq_field_dot runs on the context's stream
        self.ctx._chk(L.library().kq_field_dot(self.ctx._h, _p(x), _p(y), C.byref(out)), "kq_field_dot")
        return out.value

    def close(self):
        self.ctx.close()


def exchange_link_ghosts(slabs, transport):
    """Every rank gets the t links of the 3 slices below its slab from the rank below (once, after loading)."""
    faces = [s.link_face() for s in slabs]
    torch.cuda.synchronize()
    # a link face travels up in t only: send it as the 'hi' face, receive it as the lower ghost
    ghosts = transport.exchange([(f, f) for f in faces])
    # the received faces are ordered on torch's stream only, and kq_slab_set_link_ghosts copies on the context's
    torch.cuda.synchronize()
    for s, (glo, _) in zip(slabs, ghosts):
        s.set_link_ghosts(glo)


def dslash(slabs, transport, prec, srcs, dsts, dst_parity, pvecs=None, sigma=0.0, overlap=True):
    """dst_r = D src_r on every local slab (one halo exchange), or sigma * pvec_r - D src_r.  With overlap, the
    interior sites (which read no ghost) are computed while the faces are in flight, the boundary sites after they
    have arrived -- the reference's StartComm / bulk loop / EndComm (dirac_hisq.cpp:412-414, 452-454)."""
    faces = [s.pack(prec, x) for s, x in zip(slabs, srcs)]
    # packs, transfers and kernels are ordered on torch's current stream: no host synchronisation
    handle = transport.exchange_start(faces)
    pv = [None if pvecs is None else pvecs[k] for k in range(len(slabs))]
    if overlap:
        for k, (s, x, y) in enumerate(zip(slabs, srcs, dsts)):
            s.dslash(prec, x, None, None, y, dst_parity, pv[k], sigma, part=PART_INTERIOR)
    ghosts = transport.exchange_wait(handle)
    for k, (s, x, y, (glo, ghi)) in enumerate(zip(slabs, srcs, dsts, ghosts)):
        s.dslash(prec, x, glo, ghi, y, dst_parity, pv[k], sigma, part=PART_BOUNDARY if overlap else PART_ALL)


def _global_dot(slabs, transport, x, y) -> float:
    outs = [torch.zeros(1, dtype=torch.float64, device=f"cuda:{s.device}") for s in slabs]
    for s, xk, yk, o in zip(slabs, x, y, outs):
        s.dot_device(xk, yk, o)
    transport.allreduce_inplace(outs)
    return float(outs[0].item())


def _operator(slabs, transport, prec, p0, tmp, sv, sloppy, parity, sigma, overlap):
    """sv = sigma p0 - D_pq D_qp p0 on FP64 slab fields, the dslash in precision prec (p0 converted to it, the result
    converted back: the inexact matvec of a relaxed-precision Krylov solver)"""
    D = L.KUQCD_DOUBLE
    if prec == D:
        dslash(slabs, transport, D, p0, tmp, 1 - parity, overlap=overlap)
        dslash(slabs, transport, D, tmp, sv, parity, pvecs=p0, sigma=sigma, overlap=overlap)
        return
    ps, ts, ss = sloppy[prec]
    for k, s in enumerate(slabs):
        s.ctx.convert(p0[k], D, ps[k], prec, s.stream())
    dslash(slabs, transport, prec, ps, ts, 1 - parity, overlap=overlap)
    dslash(slabs, transport, prec, ts, ss, parity, pvecs=ps, sigma=sigma, overlap=overlap)
    for k, s in enumerate(slabs):
        s.ctx.convert(ss[k], prec, sv[k], D, s.stream())


def _cgm(slabs, transport, bs, shifts_ref, tol, max_iter, parity, overlap, poll_every, choose=None, log=None):
    ns = len(shifts_ref)
    D = L.KUQCD_DOUBLE
    vb = [s.ctx.spinor_bytes(D) for s in slabs]
    r = [s.field() for s in slabs]
    sv = [s.field() for s in slabs]
    tmp = [s.field() for s in slabs]
    pblk = [torch.zeros(ns * n, dtype=torch.uint8, device=f"cuda:{s.device}") for s, n in zip(slabs, vb)]
    xblk = [torch.zeros(ns * n, dtype=torch.uint8, device=f"cuda:{s.device}") for s, n in zip(slabs, vb)]
    p0 = [pb[:n] for pb, n in zip(pblk, vb)]
    st = [s.cgm_state() for s in slabs]
    for k, s in enumerate(slabs):
        s.cgm_init(st[k], shifts_ref, tol, max_iter)
        s.axpby(1.0, bs[k], 0.0, r[k])
        for j in range(ns):
            s.axpby(1.0, bs[k], 0.0, pblk[k][j * vb[k]:(j + 1) * vb[k]])
        s.dot_device(r[k], r[k], st[k][1:2])
    transport.allreduce_inplace([t[1:2] for t in st])
    for k, s in enumerate(slabs):
        s.cgm_step(st[k], L.KQ_CGM_START)
    it, done, rr = slabs[0].cgm_poll(st[0], with_rr=True)
    sloppy = {}
    while not done:
        prec = D if choose is None else choose(rr)
        if prec != D and prec not in sloppy:
            sloppy[prec] = tuple([s.field(prec) for s in slabs] for _ in range(3))
        for _ in range(poll_every):
            # s = shifts[0] p0 - D_pq D_qp p0 (MdaggM + Axmy, inverter_cgm.cpp:44-46)
            _operator(slabs, transport, prec, p0, tmp, sv, sloppy, parity, shifts_ref[0], overlap)
            for k, s in enumerate(slabs):
                s.dot_device(p0[k], sv[k], st[k][0:1])
            transport.allreduce_inplace([t[0:1] for t in st])
            for k, s in enumerate(slabs):
                s.cgm_step(st[k], L.KQ_CGM_ALPHA)
                s.cgm_residual(st[k], sv[k], r[k])
            transport.allreduce_inplace([t[1:2] for t in st])
            for k, s in enumerate(slabs):
                s.cgm_step(st[k], L.KQ_CGM_BETA)
                s.cgm_update(st[k], r[k], pblk[k], xblk[k])
                s.cgm_step(st[k], L.KQ_CGM_FINISH)
        it2, done, rr = slabs[0].cgm_poll(st[0], with_rr=True)
        if log is not None:
            log[prec] = log.get(prec, 0) + it2 - it
        it = it2
    torch.cuda.synchronize()
    x = [[xblk[k][j * vb[k]:(j + 1) * vb[k]] for j in range(ns)] for k in range(len(slabs))]
    return x, it


def cgm(slabs, transport, bs, shifts_ref, tol, max_iter, parity=0, overlap=True, poll_every=4):
    """Multishift CG of inverter_cgm.cpp:17-87 on FP64 slab fields.  shifts_ref: reference semantics (x_0 solves
    shifts[0] - DD, x_j solves shifts[0] + shifts[j] - DD); stops shift k when Z_k^2 |r|^2 < tol.  Returns
    (xs, iterations) with xs[r][k] the local solution of shift k on slab r.

    Device-driven: the scalar recurrences run on a device state (kq_slab_cgm_*), each of the two reductions per
    iteration is a device-side local sum and one in-place all-reduce over ranks (the reference's MPI_Allreduce,
    spinor_field.cpp:207-215, 235-243), the shift vectors are updated in one fused pass, and the two dslash overlap
    their halo exchange; everything is ordered on torch's current stream.  The host reads the state once every
    poll_every iterations (steps after the stop are no-ops, so the iteration count is the reference's)."""
    return _cgm(slabs, transport, bs, shifts_ref, tol, max_iter, parity, overlap, poll_every)


def relaxed_thresholds(rel_residual, sloppy=L.KUQCD_HALF, eps32=3e-7, eps16=1e-3, relax_frac=0.3):
    """(rho32, rho16) of the relaxed-precision schedule: the operator may run on FP32 links below |r| = rho32 |b| and
    on HALF links below rho16 |b| (0: no HALF phase), rho = relax_frac * target / eps (the single-GPU mixed
    solver's rule: a matvec error eps |A| |p| made at |r| = rho |b| perturbs the final residual by about eps rho)."""
    rho32 = relax_frac * rel_residual / eps32
    rho16 = relax_frac * rel_residual / eps16 if sloppy == L.KUQCD_HALF else 0.0
    return rho32, rho16


def relaxed_precision(rel2, rho32, rho16):
    """The operator precision for a squared relative residual |r|^2 / |b|^2."""
    if rho16 > 0.0 and rel2 < rho16 * rho16:
        return L.KUQCD_HALF
    return L.KUQCD_SINGLE if rel2 < rho32 * rho32 else L.KUQCD_DOUBLE


def cgm_mixed(slabs, transport, bs, shifts_ref, rel_residual, max_iter, parity=0, sloppy=L.KUQCD_HALF, overlap=True,
              poll_every=4, eps32=3e-7, eps16=1e-3, relax_frac=0.3, stop_frac=0.7, max_refine=4):
    """The single-GPU mixed solver's schedule over slabs: a relaxed-precision multishift CG (operator on FP64 links
    while |r| >= rho32 |b|, then FP32, then -- sloppy = HALF -- HALF below rho16 |b|, with rho = relax_frac *
    rel_residual / eps; all vectors and scalars FP64; the precision is chosen at every poll), stopped at stop_frac *
    rel_residual, then every shift's FP64 true residual |b - (sigma_k - DD) x_k| / |b| checked and, above
    rel_residual, refined by FP64 slab CG on the residual.  Returns (xs, info): info["iterations"],
    info["refine_iterations"], info["true_residuals"] (per shift) and info["iterations_by_precision"]."""
    D = L.KUQCD_DOUBLE
    bb = _global_dot(slabs, transport, bs, bs)
    rho32, rho16 = relaxed_thresholds(rel_residual, sloppy, eps32, eps16, relax_frac)

    def choose(rr):
        return relaxed_precision(rr / bb, rho32, rho16)

    log = {}
    xs, it = _cgm(slabs, transport, bs, shifts_ref, (stop_frac * rel_residual) ** 2 * bb, max_iter, parity, overlap,
                  poll_every, choose=choose, log=log)
    sig = [shifts_ref[0]] + [shifts_ref[0] + s for s in shifts_ref[1:]]
    tmp = [s.field() for s in slabs]
    res = [s.field() for s in slabs]
    refine_it, true_res = 0, []
    for k, sk in enumerate(sig):
        xk = [xr[k] for xr in xs]
        for attempt in range(max_refine + 1):
            # res = b - (sigma_k - D D) x_k in FP64
            dslash(slabs, transport, D, xk, tmp, 1 - parity, overlap=overlap)
            dslash(slabs, transport, D, tmp, res, parity, pvecs=xk, sigma=sk, overlap=overlap)
            for r, s in enumerate(slabs):
                s.axpby(1.0, bs[r], -1.0, res[r])
            rel = float(np.sqrt(max(_global_dot(slabs, transport, res, res), 0.0) / bb))
            if rel <= rel_residual or attempt == max_refine:
                break
            es, its = _cgm(slabs, transport, res, [sk], (0.5 * rel_residual) ** 2 * bb, max_iter, parity, overlap,
                           poll_every)
            refine_it += its
            for r, s in enumerate(slabs):
                s.axpby(1.0, es[r][0], 1.0, xk[r])
        true_res.append(rel)
    torch.cuda.synchronize()
    names = {L.KUQCD_DOUBLE: "double", L.KUQCD_SINGLE: "single", L.KUQCD_HALF: "half"}
    return xs, {"iterations": it, "refine_iterations": refine_it, "true_residuals": true_res,
                "iterations_by_precision": {names[p]: n for p, n in log.items()}}
