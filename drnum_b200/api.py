"""Host-side mirror of the reference operator API for the patch step.

Names, argument meaning and error behaviour follow DrNUM's host classes so a
driver written against the reference reads the same:

    reference (file:line)                              here
    -------------------------------------------------  ---------------------------
    CartesianPatch (cartesianpatch.h, patch_common.h)  CartesianPatch
    PatchGrid (patchgrid.h:45-200)                     PatchGrid.insertPatch/computeDependencies
    AusmPlus<5, Upwind2<5, VanAlbada>, PerfectGas>     AusmPlus(Upwind2(VanAlbada()), PerfectGas())
      (fluxes/ausmplus.h:29-106)
    GPU_CartesianIterator<5, OP>(op, cuda_device)      B200CartesianIterator(op, cuda_device, precision)
      (iterators/gpu_cartesianiterator.h:29-40)
    PatchIterator::addPatch/compute/computeAll/        same method names
      copyField/updateHost/updateDevice
      (iterators/patchiterator.h:28-72)
    RungeKutta::addAlpha/addIterator/operator()(dt)    RungeKutta.addAlpha/addIterator/__call__(dt)
      (rungekutta.h:28-40, timeintegration.h:33-50)

Errors: the reference prints and exits (BUG/ERROR, drnum.h:109-128); here a
failing call raises DnError with the library's message.  All numerical work
goes through the native library (libdrnum_b200.so); there is no host
fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import DN_FACE_CLOSED, DN_FACE_PERIODIC, DN_FP32, DN_FP64, check


# ----------------------------------------------------------- flux functor concept

class VanAlbada:
    """reconstruction/vanalbada.h:26-34"""


class Upwind2:
    """reconstruction/upwind2.h:26-53 (MUSCL on conservative variables)."""

    def __init__(self, limiter=None):
        self.limiter = limiter if limiter is not None else VanAlbada()


class PerfectGas:
    """perfectgas.h:26-45: R = 287.2, gamma = 1.4, cp = 1004.5, cv = 717.5."""
    R = 287.2
    gamma = 1.4
    cp = 1004.5
    cv = 717.5


class _EulerFlux:
    """An Euler face-flux functor with its reconstruction and gas model.  The
    device path implements the Upwind2<VanAlbada> reconstruction and
    PerfectGas; `scheme` is the DN_FLUX_* constant of the C ABI."""
    scheme = _lib.DN_FLUX_AUSMPLUS

    def __init__(self, reconstruction=None, gas=None):
        self.reconstruction = reconstruction if reconstruction is not None else Upwind2(VanAlbada())
        self.gas = gas if gas is not None else PerfectGas()
        if not isinstance(self.reconstruction, Upwind2) or not isinstance(self.reconstruction.limiter, VanAlbada):
            raise ValueError("the device path implements Upwind2<VanAlbada> reconstruction only")
        if not isinstance(self.gas, PerfectGas):
            raise ValueError("the device path implements PerfectGas only")


class AusmPlus(_EulerFlux):
    """AUSM+ (fluxes/ausmplus.h:29-106): the specialised fused kernels (FP64
    and FP32 bulk).  functor=True runs the same flux through the generic
    functor kernel (FP64, bitwise equal)."""

    def __init__(self, reconstruction=None, gas=None, functor=False):
        super().__init__(reconstruction, gas)
        self.scheme = _lib.DN_FLUX_AUSMPLUS_FUNCTOR if functor else _lib.DN_FLUX_AUSMPLUS


class VanLeer(_EulerFlux):
    """Van Leer flux-vector splitting (fluxes/vanleer.h:29-196), FP64,
    through the generic functor kernel."""
    scheme = _lib.DN_FLUX_VANLEER


class Roe(_EulerFlux):
    """Roe flux with the reference's entropy modification (fluxes/roe.h:
    29-661), FP64, through the generic functor kernel."""
    scheme = _lib.DN_FLUX_ROE


# ----------------------------------------------------------------------- patches

class CartesianPatch:
    """A Cartesian patch with host-side fields [field][var][i][j][k].

    Mirrors CartesianPatch's geometry accessors (sizeI/J/K, dx/dy/dz, dV),
    its field accessors (getField, f) and the active mask
    (activate/deactivate/isActive, cartesianpatch_common.h:332-334).
    Faces are periodic or closed per axis.
    """

    def __init__(self, ni, nj, nk, lengths=None, spacing=None, origin=(0.0, 0.0, 0.0),
                 periodic=(True, True, True), num_fields=3, seek=(0, 0, 0, 0, 0, 0), add_protect=0):
        self.m_NumI, self.m_NumJ, self.m_NumK = int(ni), int(nj), int(nk)
        self.lengths = (0.0, 0.0, 0.0) if lengths is None else tuple(float(x) for x in lengths)
        if spacing is None:
            if lengths is None:
                raise ValueError("give lengths or spacing")
            # CartesianPatch::computeDeltas (cartesianpatch.cpp:160-162)
            spacing = (lengths[0] / ni, lengths[1] / nj, lengths[2] / nk)
        self.m_Dx, self.m_Dy, self.m_Dz = (float(s) for s in spacing)
        self.origin = tuple(float(o) for o in origin)
        self.periodic = tuple(bool(p) for p in periodic)
        # seek layers imin..kmax and additional protected layers
        # (CartesianPatch::setSeekExceptions, cartesianpatch.cpp:146-157)
        self.seek = tuple(int(x) for x in seek)
        self.add_protect = int(add_protect)
        self.grid = None
        self.grid_index = None
        # patch-face fluxes per side: (kind, params, table), see setBoundary
        self.bcs = {}
        # level-set wall: (G, num_inner, num_outer, min_inner_rel_dist), see setLevelSet
        self.levelset = None
        self.m_NumFields = num_fields
        self.data = np.zeros((num_fields, 5, ni, nj, nk))
        self.active = np.ones((ni, nj, nk), dtype=np.uint8)

    def sizeI(self): return self.m_NumI
    def sizeJ(self): return self.m_NumJ
    def sizeK(self): return self.m_NumK
    def sizeL(self): return self.m_NumI * self.m_NumJ * self.m_NumK
    def dx(self): return self.m_Dx
    def dy(self): return self.m_Dy
    def dz(self): return self.m_Dz
    def dV(self): return self.m_Dx * self.m_Dy * self.m_Dz
    def numVariables(self): return 5
    def numFields(self): return self.m_NumFields

    def getField(self, i_field):
        return self.data[i_field]

    def f(self, i_field, i_var, i, j, k):
        return self.data[i_field, i_var, i, j, k]

    def setField(self, i_field, values):
        self.data[i_field][...] = values

    def setBoundary(self, side, kind, params=None, table=None):
        """Flux functor wall method of side 0..5 (x-min, x-max, y-min, y-max,
        z-min, z-max): DN_BC_ZERO_FLUX, DN_BC_FARFIELD (params p, T, u, v, w:
        CompressibleFarfieldFlux::setFarfield, compressiblefarfieldflux.h:87-90),
        DN_BC_SLIP (CompressibleSlipFlux) or DN_BC_INFLOW (a per-face table
        {p or NaN, T, u, v, w}, the JetFlux::xWallM form)."""
        if self.periodic[side // 2]:
            raise ValueError(f"axis {side // 2} is periodic")
        self.bcs[int(side)] = (int(kind), None if params is None else tuple(float(x) for x in params),
                               None if table is None else np.ascontiguousarray(table, dtype=np.float64))

    def setLevelSet(self, G, num_inner_layers=3, num_outer_layers=0, min_inner_rel_dist=0.1):
        """Slip wall on the zero level of the signed-distance field G
        ([ni][nj][nk]): LevelSetObject(levelset, grid, field, var, num_inner,
        num_outer, min_inner_rel_dist) + CPU_LevelSetObjectBC<LSOBCCompressibleEulerOp>
        (levelsetobject.cpp:24-41, cpu_levelsetobjectbc.h:58-90).  G = None
        removes the wall."""
        if G is None:
            self.levelset = None
            return
        G = np.ascontiguousarray(G, dtype=np.float64)
        if G.shape != (self.m_NumI, self.m_NumJ, self.m_NumK):
            raise ValueError("level-set field must have the patch's shape")
        self.levelset = (G, int(num_inner_layers), int(num_outer_layers), float(min_inner_rel_dist))

    def deactivate(self, i, j, k): self.active[i, j, k] = 0
    def activate(self, i, j, k): self.active[i, j, k] = 1
    def isActive(self, i, j, k): return bool(self.active[i, j, k])

    def desc(self) -> _lib.dn_patch_desc:
        d = _lib.dn_patch_desc()
        d.ni, d.nj, d.nk = self.m_NumI, self.m_NumJ, self.m_NumK
        for a in range(3):
            d.face[a] = DN_FACE_PERIODIC if self.periodic[a] else DN_FACE_CLOSED
        d.dx, d.dy, d.dz = self.m_Dx, self.m_Dy, self.m_Dz
        for a in range(3):
            d.origin[a] = self.origin[a]
            d.length[a] = self.lengths[a]
        for a in range(6):
            d.seek[a] = self.seek[a]
        d.add_protect = self.add_protect
        return d


# -------------------------------------------------------------------- patch grid

class PatchGrid:
    """PatchGrid (patchgrid.h:45-200): the patches of a case and their
    overlap dependencies.  computeDependencies() builds every patch's donor
    tables on the host (dn_overlap_build: receiving cells, 8-point trilinear
    donor stencils, multi-donor averaging), equal to the reference's
    PatchGrid::computeDependencies (patchgrid.cpp:119-268)."""

    def __init__(self, num_seeklayers=2, num_addprotectlayers=0):
        self.m_NumSeekLayers = int(num_seeklayers)
        self.m_NumAddProtectLayers = int(num_addprotectlayers)
        self.m_Patches: list[CartesianPatch] = []
        self.tables = None
        self.no_donor = 0

    def insertPatch(self, patch: CartesianPatch) -> int:
        patch.add_protect = self.m_NumAddProtectLayers
        patch.grid = self
        patch.grid_index = len(self.m_Patches)
        self.m_Patches.append(patch)
        self.tables = None
        return patch.grid_index

    def getNumPatches(self):
        return len(self.m_Patches)

    def readGrid(self, gridfilename, scale=1.0):
        """PatchGrid::readGrid (patchgrid.cpp:479-557) through dn_grid_read:
        inserts a closed CartesianPatch per type-1001 block of the file, with
        its seek-layer counts; returns the patches' solver-code strings."""
        lib = _lib.load()
        h = ctypes.c_void_p()
        check(None, lib.dn_grid_read(str(gridfilename).encode(), float(scale), ctypes.byref(h)))
        codes = []
        try:
            n = ctypes.c_int()
            check(None, lib.dn_gridfile_count(h, ctypes.byref(n)))
            for i in range(n.value):
                d = _lib.dn_patch_desc()
                buf = ctypes.create_string_buffer(4096)
                check(None, lib.dn_gridfile_patch(h, i, ctypes.byref(d), buf, len(buf)))
                patch = CartesianPatch(d.ni, d.nj, d.nk, lengths=tuple(d.length), spacing=(d.dx, d.dy, d.dz),
                                       origin=tuple(d.origin), periodic=(False, False, False),
                                       seek=tuple(d.seek))
                self.insertPatch(patch)
                codes.append(buf.value.decode())
        finally:
            lib.dn_gridfile_destroy(h)
        return codes

    def writeGrid(self, gridfilename, codes=None):
        """Writes the patches as a grid file (dn_grid_write; the layout of the
        reference's grid generator, Python/drnum.py:199-244)."""
        lib = _lib.load()
        arr = (_lib.dn_patch_desc * len(self.m_Patches))(*[p.desc() for p in self.m_Patches])
        cs = None
        if codes is not None:
            cs = (ctypes.c_char_p * len(codes))(*[c.encode() for c in codes])
        check(None, lib.dn_grid_write(str(gridfilename).encode(), len(self.m_Patches), arr, cs))

    def getPatch(self, i):
        return self.m_Patches[i]

    def computeDependencies(self, with_intercoeff=True):
        if not with_intercoeff:
            raise ValueError("only with_intercoeff=True is supported (patchgrid.cpp:150-153)")
        lib = _lib.load()
        arr = (_lib.dn_patch_desc * len(self.m_Patches))(*[p.desc() for p in self.m_Patches])
        h = ctypes.c_void_p()
        nd = ctypes.c_int64()
        check(None, lib.dn_overlap_build(arr, len(self.m_Patches), ctypes.byref(h), ctypes.byref(nd)))
        try:
            self.tables = [_lib.read_donor_tables(lib.dn_overlap_counts, lib.dn_overlap_get, h, p)
                           for p in range(len(self.m_Patches))]
        finally:
            lib.dn_overlap_destroy(h)
        self.no_donor = int(nd.value)
        return self.tables


# --------------------------------------------------------------------- iterator

class B200CartesianIterator:
    """Counterpart of GPU_CartesianIterator<5, OP>(op, cuda_device) for the
    B200 kernels.  `precision` selects the plain FP64 path (DN_FP64) or the
    FP32 bulk path (DN_FP32)."""

    def __init__(self, op=None, cuda_device=0, precision=DN_FP64):
        self.m_Op = op if op is not None else AusmPlus()
        if not isinstance(self.m_Op, _EulerFlux):
            raise ValueError("flux functor must be AusmPlus, VanLeer or Roe (Upwind2(VanAlbada()), PerfectGas())")
        self.lib = _lib.load()
        self.precision = precision
        self.ctx = ctypes.c_void_p()
        check(None, self.lib.dn_ctx_create(int(cuda_device), int(precision), ctypes.byref(self.ctx)))
        if self.m_Op.scheme != _lib.DN_FLUX_AUSMPLUS:
            check(self.ctx, self.lib.dn_set_flux_scheme(self.ctx, int(self.m_Op.scheme)))
        self.m_Patches: list[CartesianPatch] = []
        self.m_PatchActive: list[bool] = []
        self.m_Shadow: list[bool] = []

    def __del__(self):
        ctx = getattr(self, "ctx", None)
        if ctx:
            self.lib.dn_ctx_destroy(ctx)
            self.ctx = None

    def close(self):
        self.__del__()

    # PatchIterator interface (patchiterator.h:43-54)
    def addPatch(self, patch: CartesianPatch, shadow=False) -> int:
        """Adds a patch; shadow=True adds another rank's patch as a compact
        shadow (dn_patch_add_shadow: no field memory until dn_shadow_alloc
        gives it the donor cells this rank receives; see shard.py)."""
        pid = ctypes.c_int()
        d = patch.desc()
        add = self.lib.dn_patch_add_shadow if shadow else self.lib.dn_patch_add
        check(self.ctx, add(self.ctx, ctypes.byref(d), ctypes.byref(pid)))
        self.m_Patches.append(patch)
        self.m_PatchActive.append(True)
        self.m_Shadow.append(bool(shadow))
        return pid.value

    def isShadow(self, i):
        return self.m_Shadow[i]

    def deviceCells(self, i):
        """Cells per variable patch i holds on the device (dn_patch_device_cells)."""
        n = ctypes.c_int64()
        check(self.ctx, self.lib.dn_patch_device_cells(self.ctx, int(i), ctypes.byref(n)))
        return n.value

    def numPatches(self):
        return len(self.m_Patches)

    def getPatch(self, i):
        return self.m_Patches[i]

    def activatePatch(self, i):
        """PatchIterator::activatePatch (patchiterator.h:119-125)."""
        if not 0 <= i < len(self.m_Patches):
            raise IndexError(i)
        check(self.ctx, self.lib.dn_patch_activate(self.ctx, i, 1))
        self.m_PatchActive[i] = True

    def deactivatePatch(self, i):
        """PatchIterator::deactivatePatch (patchiterator.h:127-133): the patch
        keeps its state through later stages (dn_patch_activate)."""
        if not 0 <= i < len(self.m_Patches):
            raise IndexError(i)
        check(self.ctx, self.lib.dn_patch_activate(self.ctx, i, 0))
        self.m_PatchActive[i] = False

    def patchActive(self, i):
        return self.m_PatchActive[i]

    def setBase(self, i_patch, base, scale):
        b = np.ascontiguousarray(base, dtype=np.float64)
        s = np.ascontiguousarray(scale, dtype=np.float64)
        check(self.ctx, self.lib.dn_patch_set_base(self.ctx, i_patch, _lib.dptr(b), _lib.dptr(s)))

    def setDonorTables(self):
        """Hands the donor tables of the patches' PatchGrid to the device
        (dn_patch_set_donors); donor patch ids map through the grid."""
        for pid, p in enumerate(self.m_Patches):
            if p.grid is None or p.grid.tables is None:
                continue
            to_it = {q.grid_index: i for i, q in enumerate(self.m_Patches) if q.grid is p.grid}
            t = p.grid.tables[p.grid_index]
            dp = np.ascontiguousarray([to_it[int(d)] for d in t["donor_patch"]], dtype=np.int32)
            counts = np.ascontiguousarray(t["counts"], dtype=np.int64)
            args = [np.ascontiguousarray(t[k]) for k in ("rec_unique",)] + [dp] + \
                   [np.ascontiguousarray(t[k]) for k in ("num_receivers", "stride", "rec_concat", "donor_idx", "weight")]
            types = [c for _, _, c, _ in _lib.DONOR_FIELDS]
            check(self.ctx, self.lib.dn_patch_set_donors(self.ctx, pid, _lib.ptr(counts, ctypes.c_int64),
                                                         *[_lib.ptr(a, ct) for a, ct in zip(args, types)]))

    def setDonorTablesOf(self, i_patch, t):
        """Hands donor tables built elsewhere to patch i_patch
        (dn_patch_set_donors): a dict in the layout of donorTables(), donor
        patches given as this iterator's patch ids."""
        counts = np.ascontiguousarray(t["counts"], dtype=np.int64)
        arrs = [np.ascontiguousarray(t[name], dtype=dt) for name, dt, _, _ in _lib.DONOR_FIELDS]
        types = [c for _, _, c, _ in _lib.DONOR_FIELDS]
        check(self.ctx, self.lib.dn_patch_set_donors(self.ctx, int(i_patch), _lib.ptr(counts, ctypes.c_int64),
                                                     *[_lib.ptr(a, ct) for a, ct in zip(arrs, types)]))

    def computeDependencies(self):
        """Builds the donor tables of the iterator's patches on the context
        (dn_grid_compute_dependencies); returns the number of seek cells
        without a donor."""
        nd = ctypes.c_int64()
        check(self.ctx, self.lib.dn_grid_compute_dependencies(self.ctx, ctypes.byref(nd)))
        return nd.value

    def donorTables(self, i_patch):
        return _lib.read_donor_tables(self.lib.dn_patch_donor_counts, self.lib.dn_patch_get_donors, self.ctx, i_patch)

    def setBoundaries(self):
        """Hands every patch's side fluxes to the device (dn_patch_set_bc)."""
        for pid, p in enumerate(self.m_Patches):
            for side, (kind, params, table) in sorted(p.bcs.items()):
                pa = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
                check(self.ctx, self.lib.dn_patch_set_bc(self.ctx, pid, side, kind,
                                                         None if pa is None else _lib.dptr(pa),
                                                         None if table is None else _lib.dptr(table)))

    def setLevelSets(self):
        """Hands every patch's level-set wall to the device (dn_patch_set_levelset)."""
        for pid, p in enumerate(self.m_Patches):
            if p.levelset is None or self.m_Shadow[pid]:
                check(self.ctx, self.lib.dn_patch_set_levelset(self.ctx, pid, None, 0, 0, 0.0))
            else:
                G, ni, no, mr = p.levelset
                check(self.ctx, self.lib.dn_patch_set_levelset(self.ctx, pid, _lib.dptr(G), ni, no, mr))

    def levelSetLayers(self, i_patch):
        p = self.m_Patches[i_patch]
        if p.levelset is None:
            return None
        return _lib.read_levelset_layers(self.lib.dn_patch_levelset_count, self.lib.dn_patch_levelset_get, self.ctx,
                                         (i_patch,), p.levelset[1], p.levelset[2])

    def updateDevice(self, fields=(0, 1)):
        self.setDonorTables()
        self.setBoundaries()
        self.setLevelSets()
        for pid, p in enumerate(self.m_Patches):
            for f in fields:
                a = np.ascontiguousarray(p.data[f], dtype=np.float64)
                check(self.ctx, self.lib.dn_patch_upload(self.ctx, pid, f, _lib.dptr(a)))
            if p.active.all() or self.m_Shadow[pid]:
                check(self.ctx, self.lib.dn_patch_set_active(self.ctx, pid, None))
            else:
                m = np.ascontiguousarray(p.active, dtype=np.uint8)
                check(self.ctx, self.lib.dn_patch_set_active(self.ctx, pid, _lib.u8ptr(m)))

    def updateHost(self, fields=(0, 1)):
        """Downloads every patch but the compact shadows (another rank's)."""
        for pid, p in enumerate(self.m_Patches):
            if self.m_Shadow[pid]:
                continue
            for f in fields:
                a = np.empty(p.data[f].shape, dtype=np.float64)
                check(self.ctx, self.lib.dn_patch_download(self.ctx, pid, f, _lib.dptr(a)))
                p.data[f][...] = a

    def downloadField(self, i_patch, i_field=0):
        """Field i_field of one patch as a new [5][ni][nj][nk] array (the
        host patch is left unchanged)."""
        p = self.m_Patches[i_patch]
        a = np.empty((5, p.m_NumI, p.m_NumJ, p.m_NumK), dtype=np.float64)
        check(self.ctx, self.lib.dn_patch_download(self.ctx, i_patch, i_field, _lib.dptr(a)))
        return a

    def copyField(self, i_src, i_dst):
        check(self.ctx, self.lib.dn_copy_field(self.ctx, i_src, i_dst))

    def compute(self, factor, patches=None):
        """PatchIterator::compute(factor, patches) (patchiterator.h:50): one
        stage of the listed patches (all when None); the others keep their
        state."""
        if patches is None or list(patches) == list(range(len(self.m_Patches))):
            check(self.ctx, self.lib.dn_compute(self.ctx, float(factor)))
            return
        ids = np.ascontiguousarray(list(patches), dtype=np.int32)
        check(self.ctx, self.lib.dn_compute_patches(self.ctx, float(factor), ids.ctypes.data, len(ids)))

    def computeAll(self, factor):
        self.compute(factor)

    def copyDonorData(self, i_field):
        """PatchIterator::copyDonorData (patchiterator.h:106-111)."""
        check(self.ctx, self.lib.dn_copy_donor_data(self.ctx, int(i_field)))

    def rkStep(self, dt, alphas):
        a = np.ascontiguousarray(alphas, dtype=np.float64)
        check(self.ctx, self.lib.dn_rk_step(self.ctx, float(dt), _lib.dptr(a), len(a)))

    def sync(self):
        check(self.ctx, self.lib.dn_sync(self.ctx))

    def conservationSums(self):
        out = np.zeros(5)
        check(self.ctx, self.lib.dn_conservation_sums(self.ctx, _lib.dptr(out)))
        return out

    def computeVariableDifference(self, i_patch, i_field1, i_var1, i_field2, i_var2):
        mx, l2 = ctypes.c_double(), ctypes.c_double()
        check(self.ctx, self.lib.dn_field_difference(self.ctx, i_patch, i_field1, i_var1, i_field2, i_var2,
                                                     ctypes.byref(mx), ctypes.byref(l2)))
        return mx.value, l2.value

    def flowStats(self, i_field, dt, patches=None):
        """The reference applications' output-step diagnostics over the
        given patches (default: all): (CFL_max, rho_min, rho_max) with
        CFL = max(|u|, |u+a|, |u-a|) dt / dx per cell
        (drnumBaseFlowDemo/main.h:255-284), reduced over the patches."""
        cfl, rmin, rmax = 0.0, 1000.0, 0.0
        out = np.zeros(3)
        for p in (range(self.numPatches()) if patches is None else patches):
            check(self.ctx, self.lib.dn_flow_stats(self.ctx, p, i_field, float(dt), _lib.dptr(out)))
            cfl, rmin, rmax = max(cfl, out[0]), min(rmin, out[1]), max(rmax, out[2])
        return cfl, rmin, rmax

    def setOption(self, option, value):
        """dn_set_option: DN_OPT_BATCHED (one launch per stage over all
        patches) or DN_OPT_GRAPH (CUDA-graph replay of whole steps)."""
        check(self.ctx, self.lib.dn_set_option(self.ctx, int(option), int(value)))

    def writeData(self, i_field, base_file_name, time, count):
        """PatchGrid::writeData (patchgrid.cpp:559-578) of this iterator's
        patches: <base>_<count:06d>.dnd (dn_write_data); returns the name."""
        check(self.ctx, self.lib.dn_write_data(self.ctx, int(i_field), str(base_file_name).encode(), float(time),
                                               int(count)))
        return f"{base_file_name}_{int(count):06d}.dnd"

    def readData(self, i_field, file_name):
        """PatchGrid::readData (patchgrid.cpp:580-611) into this iterator's
        patches (dn_read_data); returns the stored time."""
        t = ctypes.c_double()
        check(self.ctx, self.lib.dn_read_data(self.ctx, int(i_field), str(file_name).encode(), ctypes.byref(t)))
        return t.value

    def setFluxScheme(self, op):
        """Selects the Euler flux functor (AusmPlus, VanLeer, Roe) of an FP64
        iterator: dn_set_flux_scheme."""
        if not isinstance(op, _EulerFlux):
            raise ValueError("flux functor must be AusmPlus, VanLeer or Roe")
        check(self.ctx, self.lib.dn_set_flux_scheme(self.ctx, int(op.scheme)))
        self.m_Op = op

    def setStageFunction(self, fn, user=None):
        """Installs a caller-written stage function (dn_set_stage_function):
        `fn` is the address of an `int fn(void* user, const dn_stage_launch*)`
        (e.g. from a shared library built on drnum_b200_functor.cuh), `user`
        an address passed through; None restores the built-in scheme."""
        check(self.ctx, self.lib.dn_set_stage_function(self.ctx, fn, user))

    def setTile(self, i_patch, shape):
        check(self.ctx, self.lib.dn_patch_set_tile(self.ctx, int(i_patch), int(shape)))

    def autotune(self, cache_path=None):
        """Measures the tile shapes on this case and picks one per patch (and,
        for FP32-bulk single-patch launches, the plane-chunk length of the
        CTAs); returns the measured cost per padded cell (ns) of each shape."""
        cost = np.zeros(_lib.DN_NUM_TILE_SHAPES)
        path = None if cache_path is None else str(cache_path).encode()
        check(self.ctx, self.lib.dn_autotune(self.ctx, path, _lib.dptr(cost)))
        return cost

    def launchCount(self):
        n = ctypes.c_int64()
        check(self.ctx, self.lib.dn_launch_count(self.ctx, ctypes.byref(n)))
        return n.value

    def tmaPatchCount(self):
        """dn_tma_patch_count: patches whose planes are staged by TMA."""
        n = ctypes.c_int64()
        check(self.ctx, self.lib.dn_tma_patch_count(self.ctx, ctypes.byref(n)))
        return n.value


class B200LevelSetObjectBC:
    """Post-operation form of the level-set wall (CPU_LevelSetObjectBC::operator(),
    cpu_levelsetobjectbc.h:58-90) for the stage-by-stage RungeKutta sequence;
    dn_rk_step applies it by itself."""

    def __init__(self, iterator, field=0):
        self.it = iterator
        self.field = int(field)

    def __call__(self):
        check(self.it.ctx, self.it.lib.dn_apply_levelset_bc(self.it.ctx, self.field))


# ------------------------------------------------------------- time integration

class RungeKutta:
    """RungeKutta (rungekutta.h:28-40, rungekutta.cpp:27-42) over
    B200CartesianIterator objects: one fused dn_rk_step per iterator when no
    post-operation is registered, else the reference's stage sequence."""

    def __init__(self):
        self.m_Alpha: list[float] = []
        self.m_Iterators: list[B200CartesianIterator] = []
        self.m_PostOperations = []

    def addAlpha(self, a):
        self.m_Alpha.append(float(a))

    def addIterator(self, it):
        self.m_Iterators.append(it)

    def addPostOperation(self, op):
        self.m_PostOperations.append(op)

    def copyDonorData(self, i_field):
        for it in self.m_Iterators:
            it.copyDonorData(i_field)

    def __call__(self, dt):
        if not self.m_PostOperations:
            for it in self.m_Iterators:
                it.rkStep(dt, self.m_Alpha)
            return
        self.copyDonorData(0)
        for it in self.m_Iterators:
            it.copyField(0, 1)
        first = True
        for a in self.m_Alpha:
            if not first:
                self.copyDonorData(0)
            first = False
            for it in self.m_Iterators:
                it.computeAll(a * dt)
            self.copyDonorData(0)
            for op in self.m_PostOperations:
                op()
