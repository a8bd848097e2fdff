"""Patch grids sharded over GPUs: one process per GPU, patches partitioned by
cell count, donor cells exchanged between ranks before every donor copy.

The reference advances all patches of a grid in one process; its RK step
(RungeKutta::operator(), rungekutta.cpp:27-42) copies donor data between
patches in memory (Patch::accessDonorDataDirect, patch.cpp:573-653).  Here
every rank knows the whole grid but owns only its share
(dn_patch_set_owned): stages, donor copies into receiving cells and the
level-set wall run on owned patches, the others are shadows.  A shadow is
either a full copy (a patch added with dn_patch_add and marked unowned) or,
with `make_sharded(..., compact=True)`, a compact shadow that holds only the
donor cells this rank's receiving cells read (dn_patch_add_shadow +
dn_shadow_alloc): device memory then scales with the rank's share of the
grid plus its halo of donor cells.  Before each
donor copy, each rank sends its peers the donor cells of its patches that
their receiving patches read and receives the ones its own receiving patches
read (dn_exchange_pack / _unpack around NCCL send/recv through
torch.distributed).  The donor copy then reads local memory and the result
equals the single-GPU step bit for bit.

`rk_step_sequence` is the step itself over an operations object, so the same
sequence drives GPU contexts (`ShardedIterator`) and, in the CPU tests, the
numpy oracle with gloo transport.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check


def partition(cells, world):
    """Greedy bin packing: patches in descending cell count (ties: lower
    index first) each to the rank with the fewest cells so far (ties: lower
    rank).  Returns owner[patch]."""
    order = sorted(range(len(cells)), key=lambda p: (-int(cells[p]), p))
    load = [0] * world
    owner = [0] * len(cells)
    for p in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[p] = r
        load[r] += int(cells[p])
    return owner


class Transport:
    """Moves the exchange buffers of one rank: for every peer with cells to
    send, `pack(field, peer, buf)` fills a send buffer; sends and receives to
    all peers go out as one batch of torch.distributed point-to-point ops
    (grouped, so NCCL cannot deadlock on their order); then
    `unpack(field, peer, buf)` drains each receive buffer.  `alloc(n)` makes
    a buffer of n elements (a CUDA tensor for NCCL, a CPU tensor for gloo)."""

    def __init__(self, rank, world, counts, alloc, pack, unpack, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.world, self.group = rank, world, group
        self.pack, self.unpack = pack, unpack
        self.peers = [q for q in range(world) if q != rank]
        self.send = {q: alloc(5 * counts[q][0]) for q in self.peers if counts[q][0]}
        self.recv = {q: alloc(5 * counts[q][1]) for q in self.peers if counts[q][1]}

    def exchange(self, field):
        dist = self.dist
        ops = []
        for q in self.peers:
            if q in self.send:
                self.pack(field, q, self.send[q])
                ops.append(dist.P2POp(dist.isend, self.send[q], q, self.group))
            if q in self.recv:
                ops.append(dist.P2POp(dist.irecv, self.recv[q], q, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for q in self.peers:
            if q in self.recv:
                self.unpack(field, q, self.recv[q])


def rk_step_sequence(ops, dt, alphas):
    """One RK step of a sharded grid in the order of the reference's
    RungeKutta::operator() with post-operations (rungekutta.cpp:27-42), the
    order dn_rk_step runs: donor copy, step-start copy, then per stage
    (after the first: donor copy again), stage, donor copy, post-operations;
    every donor copy preceded by the exchange of donor cells.  `ops` provides
    exchange(field), copy_donor_data(field), copy_field(src, dst),
    compute(factor) and post_operations()."""
    ops.exchange(0)
    ops.copy_donor_data(0)
    ops.copy_field(0, 1)
    for s, a in enumerate(alphas):
        if s > 0:
            ops.exchange(0)
            ops.copy_donor_data(0)
        ops.compute(a * dt)
        ops.exchange(0)
        ops.copy_donor_data(0)
        ops.post_operations()


def reduce_flow_stats(local, group=None):
    """Max of the CFL numbers and the density maxima, min of the density
    minima over the ranks of `group` (CPU tensors: the values are three
    doubles; gloo and NCCL groups both take them through all_reduce on the
    group's device)."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([local[0], -local[1], local[2]], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t[0]), float(-t[1]), float(t[2])


def gather_sums(local, group=None):
    """Sum of the ranks' 5-vectors, added in rank order after an
    all-gather (deterministic, unlike a reduction whose order the
    collective chooses)."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    world = dist.get_world_size(group)
    mine = torch.tensor(np.asarray(local, dtype=np.float64), device=dev)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = np.zeros(len(local))
    for t in parts:
        out = out + t.cpu().numpy()
    return out


class ShardedIterator:
    """The GPU side: a B200CartesianIterator holding every patch of the grid
    (donor tables computed for all of them), owning the patches `owner`
    assigns to this rank, with an exchange plan and the process group's
    transport.  With NCCL the buffers are device tensors; with gloo they are
    host tensors, staged through device buffers around the pack and unpack
    kernels (for ranks that share a device or hosts without NCCL).  This
    rank's GPU must be the current device."""

    def __init__(self, it, owner, rank, world, group=None):
        import torch
        self.it, self.owner, self.rank, self.world, self.group = it, list(owner), rank, world, group
        lib = it.lib
        for p in range(it.numPatches()):
            if it.isShadow(p) and self.owner[p] == rank:
                raise ValueError(f"patch {p} is owned by rank {rank} but was added as a compact shadow")
            check(it.ctx, lib.dn_patch_set_owned(it.ctx, p, 1 if self.owner[p] == rank else 0))
        own = (ctypes.c_int32 * len(self.owner))(*self.owner)
        self.ex = ctypes.c_void_p()
        check(it.ctx, lib.dn_exchange_build_ctx(it.ctx, own, rank, world, ctypes.byref(self.ex)))
        if any(it.isShadow(p) for p in range(it.numPatches())):
            # compact shadows: field memory for exactly the donor cells received
            check(it.ctx, lib.dn_shadow_alloc(it.ctx, self.ex))
        counts = {}
        for q in range(world):
            ns, nr = ctypes.c_int64(), ctypes.c_int64()
            check(it.ctx, lib.dn_exchange_counts(self.ex, q, ctypes.byref(ns), ctypes.byref(nr)))
            counts[q] = (ns.value, nr.value)
        self.counts = counts
        # the library's work goes on a stream of its own (a real stream: a null
        # handle would select the context's internal stream), made torch's
        # current stream around every exchange, so that NCCL's send waits for
        # the pack kernels and the unpack kernels wait for the receive
        self.stream = torch.cuda.Stream(torch.cuda.current_device())
        check(it.ctx, lib.dn_set_stream(it.ctx, ctypes.c_void_p(self.stream.cuda_stream)))
        dtype = torch.float64 if it.precision == _lib.DN_FP64 else torch.int32
        import torch.distributed as dist
        self.host_transport = dist.get_backend(group) != "nccl"
        self.dev_send = {q: torch.empty(5 * counts[q][0], dtype=dtype, device="cuda") for q in counts if counts[q][0]}
        self.dev_recv = {q: torch.empty(5 * counts[q][1], dtype=dtype, device="cuda") for q in counts if counts[q][1]}
        if self.host_transport:
            alloc = lambda n: torch.empty(n, dtype=dtype, pin_memory=True)   # noqa: E731
        else:
            alloc = lambda n: torch.empty(n, dtype=dtype, device="cuda")     # noqa: E731
        self.transport = Transport(rank, world, counts, alloc, self._pack, self._unpack, group)
        self.post = []
        # the exchange runs inside the library's own step, before every donor
        # copy (dn_set_exchange_hook): one dn_rk_step per step, fields rotated
        # in place, no field copy
        self._hook_error = None
        self._hook = _lib.DN_EXCHANGE_FN(self._on_donor_copy)
        check(it.ctx, lib.dn_set_exchange_hook(it.ctx, self._hook, None))

    def _on_donor_copy(self, user):
        try:
            self.exchange(_lib.DN_FIELD_DONOR_COPY)
            return 0
        except Exception as e:       # reported by the library call that ran the hook
            self._hook_error = e
            return _lib.DN_ERR_STATE

    def _pack(self, field, peer, buf):
        dev = self.dev_send[peer] if self.host_transport else buf
        check(self.it.ctx, self.it.lib.dn_exchange_pack(self.it.ctx, self.ex, field, peer,
                                                        ctypes.c_void_p(dev.data_ptr())))
        if self.host_transport:
            buf.copy_(dev)                       # waits for the pack kernel (current stream)

    def _unpack(self, field, peer, buf):
        dev = buf
        if self.host_transport:
            dev = self.dev_recv[peer]
            dev.copy_(buf)                       # on the current stream, before the unpack kernel
        check(self.it.ctx, self.it.lib.dn_exchange_unpack(self.it.ctx, self.ex, field, peer,
                                                          ctypes.c_void_p(dev.data_ptr())))

    # operations of rk_step_sequence (explicit exchanges: the hook is
    # bypassed by _HookedOps below, which leaves the exchange to it)
    def exchange(self, field):
        import torch
        with torch.cuda.stream(self.stream):
            self.transport.exchange(field)

    def copy_donor_data(self, field):
        self.it.copyDonorData(field)

    def copy_field(self, src, dst):
        self.it.copyField(src, dst)

    def compute(self, factor):
        self.it.computeAll(factor)

    def post_operations(self):
        for op in self.post:
            op()

    def addPostOperation(self, op):
        self.post.append(op)

    def rkStep(self, dt, alphas):
        """One RK step of this rank's patches.  Without post-operations the
        library runs the whole step (dn_rk_step; the level-set walls set on
        the context are its post-operations) with the exchange in its hook;
        with Python post-operations the step runs stage by stage
        (rk_step_sequence), every donor copy still preceded by the hook's
        exchange."""
        try:
            if self.post:
                rk_step_sequence(_HookedOps(self), dt, alphas)
            else:
                self.it.rkStep(dt, alphas)
        except _lib.DnError:
            if self._hook_error is not None:
                e, self._hook_error = self._hook_error, None
                raise e
            raise

    def conservationSums(self):
        """FP64 conservation sums (mass, momenta, energy) of the whole grid:
        this rank's owned patches (the context sums owned patches only),
        gathered over the ranks and added in rank order, so every rank gets
        the same bits whatever the collective's own order."""
        return gather_sums(self.it.conservationSums(), self.group)

    def flowStats(self, field, dt):
        """(CFL_max, rho_min, rho_max) of the whole grid: this rank's owned
        patches on its GPU, then a max / min all-reduce over the ranks."""
        local = self.it.flowStats(field, dt, [p for p in range(len(self.owner)) if self.owner[p] == self.rank])
        return reduce_flow_stats(local, self.group)

    def deviceCells(self):
        """Cells per variable this rank holds on its GPU (owned patches and
        shadows)."""
        return sum(self.it.deviceCells(p) for p in range(self.it.numPatches()))

    def close(self):
        if self.ex:
            self.it.lib.dn_set_exchange_hook(self.it.ctx, _lib.DN_EXCHANGE_FN(), None)
            self.it.lib.dn_exchange_destroy(self.ex)
            self.ex = None


class _HookedOps:
    """rk_step_sequence operations of a ShardedIterator whose context runs
    the exchange in its donor-copy hook: the sequence's own exchanges are
    left out."""

    def __init__(self, sh):
        self.sh = sh

    def exchange(self, field):
        pass

    def copy_donor_data(self, field):
        self.sh.copy_donor_data(field)

    def copy_field(self, src, dst):
        self.sh.copy_field(src, dst)

    def compute(self, factor):
        self.sh.compute(factor)

    def post_operations(self):
        self.sh.post_operations()


def make_sharded(objs, owner, rank, world, precision, device=0, group=None, op=None, compact=True, fields=(0,),
                 tables=None):
    """A ShardedIterator over the patches `objs` (CartesianPatch objects of one
    PatchGrid whose donor tables are computed, or with `tables`: per patch
    donor tables in the layout of donorTables(), as slab_split gives them)
    for `rank`: owned patches in full, the others as compact shadows
    (compact=True) or full copies; the host state of `fields` uploaded.  The
    process group must use NCCL and `device` must be this rank's GPU."""
    from .api import AusmPlus, B200CartesianIterator
    it = B200CartesianIterator(op if op is not None else AusmPlus(), device, precision)
    for p, cp in enumerate(objs):
        it.addPatch(cp, shadow=compact and owner[p] != rank)
    if tables is not None:
        for p, t in enumerate(tables):
            it.setDonorTablesOf(p, t)
    it.updateDevice(fields=fields)
    return ShardedIterator(it, owner, rank, world, group)


def slab_patches(U, h, slabs):
    """CartesianPatch objects of the slabs of `slab_split` over the state U
    of a patch periodic in every axis, with cell spacing h."""
    from .api import CartesianPatch
    objs = []
    for s in slabs:
        cp = CartesianPatch(*s["n"], spacing=(h, h, h), periodic=(False, True, True), num_fields=1)
        cp.setField(0, slab_state(U, s))
        objs.append(cp)
    return objs


def slab_split(n, world, halo=2):
    """Splits one patch of n = (ni, nj, nk) cells, periodic along i, into
    `world` i-slabs for as many ranks (the single-patch case of the sharded
    grid).  Slab s owns the global planes [a_s, a_{s+1}) with a_s = s*ni//world
    and carries `halo` seek planes on either side, copied before every stage
    from the neighbouring slab's owned planes (across the periodic seam for
    the first and last slab) by donor tables of weight 1.  With the
    reference's two seek layers the stencil of every owned cell (two cells
    each way along i) reads only owned or freshly copied planes, so the owned
    planes advance exactly as in the unsplit patch; the seek planes' own
    updates are overwritten by the copy.

    Returns per slab a dict: n (cells), plane0 (global plane of local plane
    0, modulo ni), owned (a, b), tables (the dn_patch_set_donors layout; donor
    patch ids are slab indices)."""
    ni, nj, nk = (int(x) for x in n)
    if world < 2:
        raise ValueError("an i-slab split needs at least two slabs")
    bounds = [s * ni // world for s in range(world + 1)]
    if min(bounds[s + 1] - bounds[s] for s in range(world)) < halo:
        raise ValueError(f"{ni} planes cannot give {world} slabs of at least {halo} planes each")
    owner_of = np.empty(ni, dtype=np.int64)
    for s in range(world):
        owner_of[bounds[s]:bounds[s + 1]] = s
    plane_cells = nj * nk
    out = []
    for s in range(world):
        a, b = bounds[s], bounds[s + 1]
        n_s = b - a + 2 * halo
        seek = list(range(halo)) + list(range(n_s - halo, n_s))
        g = [(a - halo + l) % ni for l in seek]
        donors = {}
        for l, gp in zip(seek, g):
            t = int(owner_of[gp])
            lt = (gp - (bounds[t] - halo)) % ni          # the donor slab's local plane
            donors.setdefault(t, []).append((l, lt))
        rec_unique = np.concatenate([l * plane_cells + np.arange(plane_cells, dtype=np.uint64) for l in seek])
        dp, nr, st, rc, di = [], [], [], [], []
        for t in sorted(donors):
            pairs = donors[t]
            dp.append(t)
            nr.append(len(pairs) * plane_cells)
            st.append(1)
            for l, lt in pairs:
                rc.append(l * plane_cells + np.arange(plane_cells, dtype=np.uint64))
                di.append(lt * plane_cells + np.arange(plane_cells, dtype=np.uint64))
        rc = np.concatenate(rc).astype(np.uint64)
        di = np.concatenate(di).astype(np.uint64)
        tables = {"rec_unique": rec_unique.astype(np.uint64), "donor_patch": np.asarray(dp, dtype=np.int32),
                  "num_receivers": np.asarray(nr, dtype=np.int64), "stride": np.asarray(st, dtype=np.int32),
                  "rec_concat": rc, "donor_idx": di, "weight": np.ones(len(di), dtype=np.float64)}
        tables["counts"] = np.array([len(rec_unique), len(dp), len(rc), len(di)], dtype=np.int64)
        out.append({"n": (n_s, nj, nk), "plane0": (a - halo) % ni, "owned": (a, b), "tables": tables})
    return out


def slab_state(U, slab):
    """The state [5][ni][nj][nk] of one slab of `slab_split`, cut from the
    whole patch's state U (planes wrapped across the periodic seam)."""
    ni = U.shape[1]
    planes = [(slab["plane0"] + l) % ni for l in range(slab["n"][0])]
    return np.ascontiguousarray(U[:, planes])


def slab_owned(U_slab, slab, halo=2):
    """The owned planes of a slab's state."""
    a, b = slab["owned"]
    return U_slab[:, halo:halo + (b - a)]
