"""Patch grids sharded over ranks (drnum_b200/shard.py, dn_exchange_*).

CPU: the partition, the exchange lists (host-only dn_exchange_build from
the library's own donor tables), and the whole sharded RK step sequence with
gloo transport between two and three processes, each advancing its patches
with the oracle: the result equals the reference's single-process grid run
(golden fixtures) bit for bit.  GPU (one device): two contexts in one
process play two ranks, the exchange buffers handed over directly (no
kernel waits on another); the result equals one context bit for bit."""
import ctypes
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import cases_def
import pyoracle
from drnum_b200 import _lib, cases, shard
from test_overlap import TABLE_KEYS, _descs, _fixture, _ls_tables


def exchange_lists(patches, owner, rank, world):
    """(send, recv) per peer: arrays of (patch, cell) from dn_exchange_build."""
    lib = _lib.load()
    h = ctypes.c_void_p()
    nd = ctypes.c_int64()
    assert lib.dn_overlap_build(_descs(patches), len(patches), ctypes.byref(h), ctypes.byref(nd)) == _lib.DN_OK
    ex = ctypes.c_void_p()
    own = (ctypes.c_int32 * len(owner))(*owner)
    try:
        assert lib.dn_exchange_build(h, own, rank, world, ctypes.byref(ex)) == _lib.DN_OK
        out = {}
        for q in range(world):
            ns, nr = ctypes.c_int64(), ctypes.c_int64()
            assert lib.dn_exchange_counts(ex, q, ctypes.byref(ns), ctypes.byref(nr)) == _lib.DN_OK
            sp, sc = np.zeros(ns.value, np.int32), np.zeros(ns.value, np.uint64)
            rp, rc = np.zeros(nr.value, np.int32), np.zeros(nr.value, np.uint64)
            assert lib.dn_exchange_get(ex, q, sp.ctypes.data, sc.ctypes.data, rp.ctypes.data,
                                       rc.ctypes.data) == _lib.DN_OK
            out[q] = ((sp, sc), (rp, rc))
        return out
    finally:
        if ex:
            lib.dn_exchange_destroy(ex)
        lib.dn_overlap_destroy(h)


def test_partition_balances_cells():
    cells = [100, 90, 80, 70, 60, 10, 10, 10]
    owner = shard.partition(cells, 3)
    loads = [sum(c for c, o in zip(cells, owner) if o == r) for r in range(3)]
    assert owner == shard.partition(cells, 3)
    assert max(loads) - min(loads) <= 40
    assert shard.partition(cells, 1) == [0] * len(cells)


@pytest.mark.parametrize("name,world", [("octants_8", 3), ("random6", 2), ("octants_ragged", 4)])
def test_exchange_lists_pair_up_and_cover_every_remote_donor(golden_dir, name, world):
    patches = cases_def.grid_layout(name)
    owner = shard.partition([int(np.prod(p["n"])) for p in patches], world)
    lists = [exchange_lists(patches, owner, r, world) for r in range(world)]
    z = _fixture(golden_dir, name)
    for r in range(world):
        for q in range(world):
            if q == r:
                assert len(lists[r][q][0][0]) == 0 and len(lists[r][q][1][0]) == 0
                continue
            (sp, sc), _ = lists[r][q]
            _, (rp, rc) = lists[q][r]
            assert np.array_equal(sp, rp) and np.array_equal(sc, rc)
        # every donor cell a receiving patch of r reads from another rank arrives
        need = set()
        for p in range(len(patches)):
            if owner[p] != r:
                continue
            donors = z[f"p{p}_donor_patch"]
            nrec, stride, idx = z[f"p{p}_num_receivers"], z[f"p{p}_stride"], z[f"p{p}_donor_idx"]
            pos = 0
            for d, m, s in zip(donors, nrec, stride):
                n = int(m) * int(s)
                if owner[int(d)] != r:
                    need.update((int(d), int(c)) for c in idx[pos:pos + n])
                pos += n
        got = set()
        for q in range(world):
            _, (rp, rc) = lists[r][q]
            got.update(zip(rp.tolist(), rc.tolist()))
        assert got == need


def test_exchange_rejects_bad_owner():
    lib = _lib.load()
    patches = cases_def.grid_layout("pair_x")
    h = ctypes.c_void_p()
    nd = ctypes.c_int64()
    assert lib.dn_overlap_build(_descs(patches), 2, ctypes.byref(h), ctypes.byref(nd)) == _lib.DN_OK
    ex = ctypes.c_void_p()
    try:
        assert lib.dn_exchange_build(h, (ctypes.c_int32 * 2)(0, 2), 0, 2, ctypes.byref(ex)) == _lib.DN_ERR_ARG
        assert lib.dn_exchange_build(h, (ctypes.c_int32 * 2)(0, 1), 2, 2, ctypes.byref(ex)) == _lib.DN_ERR_ARG
    finally:
        lib.dn_overlap_destroy(h)


# ------------------------------------------------------------- gloo ranks on CPU

class OracleShard:
    """rk_step_sequence operations over the numpy oracle for one rank: owned
    patches advance, the others are shadows refreshed by the exchange."""

    def __init__(self, rank, world, name, golden_dir, group):
        import torch
        self.rank = rank
        z = _fixture(golden_dir, name)
        patches, states, spacings, dt, steps = cases_def.grid_case(name)
        self.patches, self.spacings, self.dt, self.steps = patches, spacings, dt, steps
        self.U = [np.ascontiguousarray(s, dtype=np.float64).copy() for s in states]
        self.owner = shard.partition([int(np.prod(p["n"])) for p in patches], world)
        empty = {k: z[f"p0_{k}"][:0] for k in TABLE_KEYS}
        self.tables = [{k: z[f"p{p}_{k}"] for k in TABLE_KEYS} if self.owner[p] == rank else empty
                       for p in range(len(patches))]
        self.bcs = cases_def.grid_bcs(name) or {}
        layers = _ls_tables(z, name, len(patches)) if name in cases_def.LEVELSET else None
        self.layers = None if layers is None else [L if self.owner[p] == rank else None for p, L in enumerate(layers)]
        lists = exchange_lists(patches, self.owner, rank, world)
        self.lists = lists
        counts = {q: (len(lists[q][0][1]), len(lists[q][1][1])) for q in range(world)}
        self.transport = shard.Transport(rank, world, counts, lambda n: torch.zeros(n, dtype=torch.float64),
                                         self._pack, self._unpack, group)

    def _pack(self, field, peer, buf):
        sp, sc = self.lists[peer][0]
        out = buf.numpy().reshape(5, -1)
        for t, (p, c) in enumerate(zip(sp, sc)):
            out[:, t] = self.U[int(p)].reshape(5, -1)[:, int(c)]

    def _unpack(self, field, peer, buf):
        rp, rc = self.lists[peer][1]
        inp = buf.numpy().reshape(5, -1)
        for t, (p, c) in enumerate(zip(rp, rc)):
            self.U[int(p)].reshape(5, -1)[:, int(c)] = inp[:, t]

    def exchange(self, field):
        self.transport.exchange(field)

    def copy_donor_data(self, field):
        pyoracle.oracle_donor_copy(self.U, self.tables)

    def copy_field(self, src, dst):
        self.Un = [u.copy() for u in self.U]

    def compute(self, factor):
        for p, u in enumerate(self.U):
            if self.owner[p] != self.rank:
                continue
            hx, hy, hz = self.spacings[p]
            res = pyoracle.oracle_residual_bc(u, (hx, hy, hz), self.bcs.get(p, {}))
            self.U[p] = self.Un[p] + (factor / (hx * hy * hz)) * res

    def post_operations(self):
        if self.layers is not None:
            pyoracle.oracle_levelset_bc(self.U, self.layers)


def _gloo_rank(rank, world, port, name, golden_dir, result_path):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        s = OracleShard(rank, world, name, golden_dir, None)
        for _ in range(s.steps):
            shard.rk_step_sequence(s, s.dt, cases_def.ALPHA)
        mine = {p: s.U[p] for p in range(len(s.U)) if s.owner[p] == rank}
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            np.savez(result_path, **{f"p{p}": u for p, u in merged.items()})
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name,world", [("octants_jet", 2), ("octants_8", 3), ("sphere_pair", 2)])
def test_sharded_rk_steps_over_gloo_equal_reference(golden_dir, tmp_path, name, world):
    z = _fixture(golden_dir, name)
    result = str(tmp_path / "sharded.npz")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, name, golden_dir, result)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    out = np.load(result)
    for p in range(int(z["num_patches"])):
        assert np.array_equal(out[f"p{p}"], z[f"p{p}_out"]), (name, p)


def _gloo_stats_rank(rank, world, port, result_path):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        local = (0.1 * (rank + 1), 1.0 - 0.01 * rank, 1.0 + 0.02 * (world - rank))
        out = shard.reduce_flow_stats(local)
        sums = shard.gather_sums(np.arange(5, dtype=np.float64) * (rank + 1) + 0.1)
        if rank == 0:
            np.save(result_path, np.concatenate([np.array(out), sums]))
    finally:
        dist.destroy_process_group()


def test_flow_stats_and_sums_reduce_over_gloo_ranks(tmp_path):
    world = 3
    result = str(tmp_path / "stats.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_gloo_stats_rank, args=(r, world, port, result)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    out = np.load(result)
    assert out[:3].tolist() == [0.1 * world, 1.0 - 0.01 * (world - 1), 1.0 + 0.02 * world]
    want = np.zeros(5)
    for r in range(world):
        want = want + (np.arange(5, dtype=np.float64) * (r + 1) + 0.1)
    assert np.array_equal(out[3:], want)


# ------------------------------------------------------------- two contexts, one GPU

class _Recorder:
    """Records the operation sequence of one RK step."""

    def __init__(self):
        self.ops = []

    def __getattr__(self, name):
        return lambda *args: self.ops.append((name, args))


@pytest.mark.gpu
@pytest.mark.parametrize("compact", [False, True])
@pytest.mark.parametrize("precision", [_lib.DN_FP64, _lib.DN_FP32])
@pytest.mark.parametrize("name", ["octants_jet", "sphere_pair"])
def test_two_contexts_as_two_ranks_equal_one_context(golden_dir, name, precision, compact):
    # compact: every rank holds its own patches and, of the others, only the
    # donor cells its receiving cells read (dn_patch_add_shadow, dn_shadow_alloc)
    import torch
    from drnum_b200.api import B200LevelSetObjectBC
    from test_gpu_grid import make_grid
    world = 2
    one, objs1, _, dt, steps = make_grid(name, precision)
    post1 = [B200LevelSetObjectBC(one)] if name in cases_def.LEVELSET else []
    patches = cases_def.grid_layout(name)
    owner = shard.partition([int(np.prod(p["n"])) for p in patches], world)
    assert len(set(owner)) == world
    ranks = [make_grid(name, precision, shadows=[compact and owner[p] != r for p in range(len(patches))])
             for r in range(world)]
    its = [r[0] for r in ranks]
    lib = _lib.load()
    exs, bufs = [], {}
    dtype = torch.float64 if precision == _lib.DN_FP64 else torch.int32
    for r, it in enumerate(its):
        for p in range(len(patches)):
            assert lib.dn_patch_set_owned(it.ctx, p, int(owner[p] == r)) == _lib.DN_OK
        ex = ctypes.c_void_p()
        own = (ctypes.c_int32 * len(owner))(*owner)
        assert lib.dn_exchange_build_ctx(it.ctx, own, r, world, ctypes.byref(ex)) == _lib.DN_OK
        if compact:
            assert lib.dn_shadow_alloc(it.ctx, ex) == _lib.DN_OK
            held = [it.deviceCells(p) for p in range(len(patches))]
            full = [one.deviceCells(p) for p in range(len(patches))]
            for p in range(len(patches)):
                if owner[p] == r:
                    assert held[p] == full[p]
                else:
                    assert held[p] < full[p], (p, held[p], full[p])   # donor cells only
            assert sum(held[p] for p in range(len(patches)) if owner[p] != r) > 0
            # a compact shadow is another rank's: its whole state stays out of reach
            q = next(p for p in range(len(patches)) if owner[p] != r)
            assert lib.dn_patch_download(it.ctx, q, 0, _lib.dptr(np.empty(5 * int(np.prod(patches[q]["n"]))))) \
                == _lib.DN_ERR_STATE
            assert lib.dn_patch_set_owned(it.ctx, q, 1) == _lib.DN_ERR_STATE
        exs.append(ex)
        for q in range(world):
            ns, nr = ctypes.c_int64(), ctypes.c_int64()
            assert lib.dn_exchange_counts(ex, q, ctypes.byref(ns), ctypes.byref(nr)) == _lib.DN_OK
            if ns.value:
                bufs[(r, q)] = torch.empty(5 * ns.value, dtype=dtype, device="cuda")
    assert bufs, "the partition leaves no donor cell to exchange"
    posts = [[B200LevelSetObjectBC(it)] if name in cases_def.LEVELSET else [] for it in its]

    def apply(r, op, args):
        it = its[r]
        if op == "copy_donor_data":
            it.copyDonorData(*args)
        elif op == "copy_field":
            it.copyField(*args)
        elif op == "compute":
            it.computeAll(*args)
        elif op == "post_operations":
            for f in posts[r]:
                f()

    rec = _Recorder()
    shard.rk_step_sequence(rec, dt, cases.RK3_ALPHA)
    for _ in range(steps):
        for op, args in rec.ops:
            if op == "exchange":
                for (r, q), b in bufs.items():
                    assert lib.dn_exchange_pack(its[r].ctx, exs[r], args[0], q, ctypes.c_void_p(b.data_ptr())) == 0
                for it in its:
                    it.sync()
                for (r, q), b in bufs.items():
                    assert lib.dn_exchange_unpack(its[q].ctx, exs[q], args[0], r, ctypes.c_void_p(b.data_ptr())) == 0
                for it in its:
                    it.sync()
            else:
                for r in range(world):
                    apply(r, op, args)
        # the same step on one context (its own stage sequence)
        one.copyDonorData(0)
        one.copyField(0, 1)
        for s, a in enumerate(cases.RK3_ALPHA):
            if s > 0:
                one.copyDonorData(0)
            one.computeAll(a * dt)
            one.copyDonorData(0)
            for f in post1:
                f()
    one.updateHost(fields=(0,))
    for it in its:
        it.updateHost(fields=(0,))
    for p in range(len(patches)):
        got = ranks[owner[p]][1][p].getField(0)
        assert np.array_equal(got, objs1[p].getField(0)), (name, p)
    if precision == _lib.DN_FP64:
        z = _fixture(golden_dir, name)
        for p in range(len(patches)):
            assert np.array_equal(ranks[owner[p]][1][p].getField(0), z[f"p{p}_out"]), (name, p)
    for ex in exs:
        lib.dn_exchange_destroy(ex)
    for it in its + [one]:
        it.close()


@pytest.mark.gpu
def test_sharded_iterator_single_rank_nccl_equals_reference(golden_dir):
    # the GPU driver class end to end on one rank (NCCL group of one): owned
    # flags, exchange plan, torch stream, the step sequence
    import datetime
    import torch
    import torch.distributed as dist
    from drnum_b200.api import B200LevelSetObjectBC
    from test_gpu_grid import make_grid
    name = "sphere_pair"
    z = _fixture(golden_dir, name)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        it, objs, _, dt, steps = make_grid(name, _lib.DN_FP64)
        sh = shard.ShardedIterator(it, [0] * len(objs), 0, 1)
        sh.addPostOperation(B200LevelSetObjectBC(it))
        for _ in range(steps):
            sh.rkStep(dt, cases.RK3_ALPHA)
        it.updateHost(fields=(0,))
        for p, cp in enumerate(objs):
            assert np.array_equal(cp.getField(0), z[f"p{p}_out"]), p
        # the grid's diagnostics and sums through the NCCL collectives equal the local ones
        assert sh.flowStats(0, dt) == it.flowStats(0, dt)
        assert np.array_equal(sh.conservationSums(), it.conservationSums())
        sh.close()
        it.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_lib.DN_FP64, _lib.DN_FP32])
def test_rank_without_owned_patches_steps_without_error(precision):
    # a rank whose share of the grid is empty (more ranks than patches): the
    # batched step has no work item and launches no stage kernel (the
    # patches are shadows, filled only by the exchange)
    from test_gpu_grid import make_grid
    it, objs, _, dt, _ = make_grid("octants_jet", precision)
    lib = _lib.load()
    for p in range(len(objs)):
        assert lib.dn_patch_set_owned(it.ctx, p, 0) == _lib.DN_OK
    l0 = it.launchCount()
    it.rkStep(dt, cases.RK3_ALPHA)
    it.sync()
    # at most the donor copies of the step (one per copy, nothing to receive)
    assert it.launchCount() - l0 <= 1 + 2 * len(cases.RK3_ALPHA)
    it.close()


# ---------------------------------------------------------------- i-slab split

def _slab_oracle_run(U0, h, dt, steps, slabs):
    """The slabs of shard.slab_split advanced with the oracle's residual
    (closed x axis, periodic y and z) and the numpy donor copy, in the order
    of RungeKutta::operator() (rungekutta.cpp:27-42)."""
    U = [shard.slab_state(U0, s) for s in slabs]
    tables = [s["tables"] for s in slabs]
    for _ in range(steps):
        pyoracle.oracle_donor_copy(U, tables)
        Un = [u.copy() for u in U]
        for q, a in enumerate(cases.RK3_ALPHA):
            if q > 0:
                pyoracle.oracle_donor_copy(U, tables)
            for p, u in enumerate(U):
                res = pyoracle.oracle_residual_bc(u, h, {}, periodic=(False, True, True))
                U[p] = Un[p] + (a * dt) / (h * h * h) * res
            pyoracle.oracle_donor_copy(U, tables)
    return U


@pytest.mark.parametrize("world", [2, 3])
def test_slab_split_tables_reproduce_the_unsplit_patch(world):
    # one periodic patch cut into i-slabs with two seek planes per side:
    # the owned planes advance bit for bit as in the unsplit patch (oracle)
    U0, h, dt = cases.periodic_box(12)
    steps = 2
    ref = pyoracle.oracle_run(U0, h, dt, steps)
    slabs = shard.slab_split(U0.shape[1:], world)
    got = _slab_oracle_run(U0, h, dt, steps, slabs)
    for s, u in zip(slabs, got):
        a, b = s["owned"]
        assert np.array_equal(shard.slab_owned(u, s), ref[:, a:b]), s["owned"]
    assert sum(s["owned"][1] - s["owned"][0] for s in slabs) == 12


def test_slab_split_rejects_thin_slabs():
    with pytest.raises(ValueError):
        shard.slab_split((5, 4, 4), 3)
    with pytest.raises(ValueError):
        shard.slab_split((8, 4, 4), 1)


def _slab_context(U0, h, slabs, which, precision, compact_owner=None, base=None):
    """A context holding the slabs `which` (the others as compact shadows
    when compact_owner is given: slab p is owned by compact_owner[p])."""
    from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch
    it = B200CartesianIterator(AusmPlus(), 0, precision)
    objs = []
    for p, s in enumerate(slabs):
        cp = CartesianPatch(*s["n"], spacing=(h, h, h), periodic=(False, True, True))
        cp.setField(0, shard.slab_state(U0, s))
        it.addPatch(cp, shadow=compact_owner is not None and compact_owner[p] != which)
        objs.append(cp)
    for p, s in enumerate(slabs):
        t = s["tables"]
        it.setDonorTablesOf(p, t)
        if base is not None:
            it.setBase(p, *base)
    it.updateDevice(fields=(0,))
    return it, objs


def _fx_base(U0):
    # one fixed-point base and range for the unsplit patch and every slab:
    # the mean state and four times the variables' magnitude scales (density,
    # rho (|u| + a) for the momenta, total energy), as a first upload derives
    # them for a patch
    U = U0.reshape(5, -1)
    base = U.mean(axis=1)
    r = U[0]
    q2 = (U[1] ** 2 + U[2] ** 2 + U[3] ** 2) / r ** 2
    T = (U[4] / r - 0.5 * q2) / 717.5
    mm = (r * (np.sqrt(q2) + np.sqrt(1.4 * 287.2 * T))).max()
    return base, 4.0 * np.array([np.abs(r).max(), mm, mm, mm, np.abs(U[4]).max()])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_lib.DN_FP64, _lib.DN_FP32])
def test_slab_split_on_one_context_equals_unsplit_patch(precision):
    from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch
    n, world, steps = 32, 3, 4
    U0, h, dt = cases.periodic_box(n)
    base = _fx_base(U0) if precision == _lib.DN_FP32 else None
    one = B200CartesianIterator(AusmPlus(), 0, precision)
    cp = CartesianPatch(n, n, n, spacing=(h, h, h))
    cp.setField(0, U0)
    one.addPatch(cp)
    if base is not None:
        one.setBase(0, *base)
    one.updateDevice(fields=(0,))
    for _ in range(steps):
        one.rkStep(dt, cases.RK3_ALPHA)
    ref = one.downloadField(0)
    one.close()
    slabs = shard.slab_split((n, n, n), world)
    it, _ = _slab_context(U0, h, slabs, 0, precision, base=base)
    for _ in range(steps):
        it.rkStep(dt, cases.RK3_ALPHA)
    for p, s in enumerate(slabs):
        a, b = s["owned"]
        assert np.array_equal(shard.slab_owned(it.downloadField(p), s), ref[:, a:b]), (p, s["owned"])
    it.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_lib.DN_FP64, _lib.DN_FP32])
def test_slab_split_over_two_contexts_with_compact_shadows(precision):
    # two contexts play two ranks of a 32^3 patch split into two slabs; each
    # holds its slab and the two seek-plane sources of the other as a compact
    # shadow; the exchange buffers are handed over between launches
    import torch
    from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch
    n, world, steps = 32, 2, 3
    U0, h, dt = cases.periodic_box(n)
    base = _fx_base(U0) if precision == _lib.DN_FP32 else None
    one = B200CartesianIterator(AusmPlus(), 0, precision)
    cp = CartesianPatch(n, n, n, spacing=(h, h, h))
    cp.setField(0, U0)
    one.addPatch(cp)
    if base is not None:
        one.setBase(0, *base)
    one.updateDevice(fields=(0,))
    for _ in range(steps):
        one.rkStep(dt, cases.RK3_ALPHA)
    ref = one.downloadField(0)
    one.close()
    slabs = shard.slab_split((n, n, n), world)
    owner = list(range(world))
    lib = _lib.load()
    its, exs, bufs = [], [], {}
    dtype = torch.float64 if precision == _lib.DN_FP64 else torch.int32
    for r in range(world):
        it, _ = _slab_context(U0, h, slabs, r, precision, compact_owner=owner, base=base)
        for p in range(world):
            assert lib.dn_patch_set_owned(it.ctx, p, int(owner[p] == r)) == _lib.DN_OK
        ex = ctypes.c_void_p()
        own = (ctypes.c_int32 * world)(*owner)
        assert lib.dn_exchange_build_ctx(it.ctx, own, r, world, ctypes.byref(ex)) == _lib.DN_OK
        assert lib.dn_shadow_alloc(it.ctx, ex) == _lib.DN_OK
        q = 1 - r
        # the shadow holds the neighbour's two planes on each side: 4 of its 20 planes
        assert it.deviceCells(q) == 4 * n * n
        for peer in range(world):
            ns, nr = ctypes.c_int64(), ctypes.c_int64()
            assert lib.dn_exchange_counts(ex, peer, ctypes.byref(ns), ctypes.byref(nr)) == _lib.DN_OK
            if ns.value:
                bufs[(r, peer)] = torch.empty(5 * ns.value, dtype=dtype, device="cuda")
        its.append(it)
        exs.append(ex)
    rec = _Recorder()
    shard.rk_step_sequence(rec, dt, cases.RK3_ALPHA)
    for _ in range(steps):
        for op, args in rec.ops:
            if op == "exchange":
                for (r, q), b in bufs.items():
                    assert lib.dn_exchange_pack(its[r].ctx, exs[r], args[0], q, ctypes.c_void_p(b.data_ptr())) == 0
                for it in its:
                    it.sync()
                for (r, q), b in bufs.items():
                    assert lib.dn_exchange_unpack(its[q].ctx, exs[q], args[0], r, ctypes.c_void_p(b.data_ptr())) == 0
                for it in its:
                    it.sync()
            elif op == "copy_donor_data":
                for it in its:
                    it.copyDonorData(*args)
            elif op == "copy_field":
                for it in its:
                    it.copyField(*args)
            elif op == "compute":
                for it in its:
                    it.computeAll(*args)
    for r, s in enumerate(slabs):
        a, b = s["owned"]
        assert np.array_equal(shard.slab_owned(its[r].downloadField(r), s), ref[:, a:b]), r
    for it, ex in zip(its, exs):
        lib.dn_exchange_destroy(ex)
        it.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_lib.DN_FP64, _lib.DN_FP32])
@pytest.mark.parametrize("name", ["octants_jet", "sphere_pair"])
def test_exchange_hook_steps_in_two_threads_equal_one_context(golden_dir, name, precision):
    # two contexts with compact shadows play two ranks, each stepping with
    # dn_rk_step in a host thread of its own; the exchange hook packs the
    # donor cells, the two threads meet at a host barrier, and each unpacks
    # the other's packed buffer (kernels never wait on one another)
    import threading
    import torch
    from test_gpu_grid import make_grid
    world = 2
    one, objs1, _, dt, steps = make_grid(name, precision)
    for _ in range(steps):
        one.rkStep(dt, cases.RK3_ALPHA)
    one.updateHost(fields=(0,))
    patches = cases_def.grid_layout(name)
    owner = shard.partition([int(np.prod(p["n"])) for p in patches], world)
    ranks = [make_grid(name, precision, shadows=[owner[p] != r for p in range(len(patches))]) for r in range(world)]
    its = [r[0] for r in ranks]
    lib = _lib.load()
    dtype = torch.float64 if precision == _lib.DN_FP64 else torch.int32
    exs, send = [], {}
    for r, it in enumerate(its):
        for p in range(len(patches)):
            assert lib.dn_patch_set_owned(it.ctx, p, int(owner[p] == r)) == _lib.DN_OK
        ex = ctypes.c_void_p()
        own = (ctypes.c_int32 * len(owner))(*owner)
        assert lib.dn_exchange_build_ctx(it.ctx, own, r, world, ctypes.byref(ex)) == _lib.DN_OK
        assert lib.dn_shadow_alloc(it.ctx, ex) == _lib.DN_OK
        ns, nr = ctypes.c_int64(), ctypes.c_int64()
        assert lib.dn_exchange_counts(ex, 1 - r, ctypes.byref(ns), ctypes.byref(nr)) == _lib.DN_OK
        send[r] = torch.empty(max(1, 5 * ns.value), dtype=dtype, device="cuda")
        exs.append(ex)
    meet = threading.Barrier(world, timeout=60)
    calls = [0, 0]

    def make_hook(r):
        def hook(user):
            it, ex, q = its[r], exs[r], 1 - r
            if lib.dn_exchange_pack(it.ctx, ex, _lib.DN_FIELD_DONOR_COPY, q, ctypes.c_void_p(send[r].data_ptr())):
                return -1
            if lib.dn_sync(it.ctx):
                return -1
            meet.wait()
            if lib.dn_exchange_unpack(it.ctx, ex, _lib.DN_FIELD_DONOR_COPY, q, ctypes.c_void_p(send[q].data_ptr())):
                return -1
            if lib.dn_sync(it.ctx):
                return -1
            meet.wait()            # both unpacked before either packs again
            calls[r] += 1
            return 0
        return _lib.DN_EXCHANGE_FN(hook)

    hooks = [make_hook(r) for r in range(world)]
    for r in range(world):
        assert lib.dn_set_exchange_hook(its[r].ctx, hooks[r], None) == _lib.DN_OK
    status = [None, None]

    def run(r):
        try:
            for _ in range(steps):
                its[r].rkStep(dt, cases.RK3_ALPHA)
            its[r].sync()
            status[r] = "ok"
        except Exception as e:      # noqa: BLE001
            status[r] = repr(e)
            meet.abort()

    threads = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert status == ["ok", "ok"], status
    assert calls == [2 * len(cases.RK3_ALPHA) * steps] * world
    for it in its:
        it.updateHost(fields=(0,))
    for p in range(len(patches)):
        assert np.array_equal(ranks[owner[p]][1][p].getField(0), objs1[p].getField(0)), (name, p)
    # outside the hook the donor-copy field is refused
    assert lib.dn_exchange_pack(its[0].ctx, exs[0], _lib.DN_FIELD_DONOR_COPY, 1,
                                ctypes.c_void_p(send[0].data_ptr())) == _lib.DN_ERR_STATE
    for r in range(world):
        lib.dn_set_exchange_hook(its[r].ctx, _lib.DN_EXCHANGE_FN(), None)
        lib.dn_exchange_destroy(exs[r])
        its[r].close()
    one.close()


def _gloo_gpu_rank(rank, world, port, name, precision, result_path):
    # one rank of a sharded grid on the shared GPU: compact shadows, the
    # library's step with the exchange in its hook, gloo between the ranks
    # (host-staged buffers; no kernel waits on another process)
    import datetime
    import torch
    import torch.distributed as dist
    from test_gpu_grid import make_grid_objects
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        objs, dt, steps = make_grid_objects(name)
        owner = shard.partition([int(np.prod(cp.data.shape[2:])) for cp in objs], world)
        sh = shard.make_sharded(objs, owner, rank, world, precision, 0)
        for _ in range(steps):
            sh.rkStep(dt, cases.RK3_ALPHA)
        sh.it.updateHost(fields=(0,))
        sums = sh.conservationSums()
        held = sh.deviceCells()
        mine = {f"p{p}": objs[p].getField(0) for p in range(len(objs)) if owner[p] == rank}
        np.savez(f"{result_path}.{rank}.npz", sums=sums, held=held, **mine)
        sh.close()
        sh.it.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_lib.DN_FP64, _lib.DN_FP32])
@pytest.mark.parametrize("name", ["octants_jet", "sphere_pair"])
def test_sharded_processes_on_one_gpu_equal_one_context(tmp_path, name, precision):
    # two processes play two ranks end to end through shard.make_sharded
    # (partition, compact shadows, exchange in the step's hook, gathered
    # sums), their buffers moved by gloo through the host
    from test_gpu_grid import make_grid
    world = 2
    one, objs1, _, dt, steps = make_grid(name, precision)
    for _ in range(steps):
        one.rkStep(dt, cases.RK3_ALPHA)
    one.updateHost(fields=(0,))
    sums1 = one.conservationSums()
    total = sum(one.deviceCells(p) for p in range(len(objs1)))
    one.close()
    result = str(tmp_path / "rank")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_gloo_gpu_rank, args=(r, world, port, name, precision, result)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    seen = set()
    for r in range(world):
        z = np.load(f"{result}.{r}.npz")
        for k in z.files:
            if k.startswith("p"):
                p = int(k[1:])
                assert np.array_equal(z[k], objs1[p].getField(0)), (name, p)
                seen.add(p)
        # the grid's sums, gathered in rank order: the single context's up to
        # the order of the per-patch additions
        assert np.allclose(z["sums"], sums1, rtol=1e-13, atol=0.0)
        assert int(z["held"]) < total
    assert seen == set(range(len(objs1)))
