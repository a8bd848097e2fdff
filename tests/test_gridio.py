"""Grid files (dn_grid_read / dn_grid_write) against the reference's own
PatchGrid::readGrid (compiled reference), and the .dnd restart format.

Grid files: the same file read by both gives the same cells, reference
points, spacings and solver-code strings, and the same donor tables after
computeDependencies (which checks the seek-layer counts).  .dnd files: the
reference writes them through Qt's QDataStream, which is not in this image,
so the format is pinned to QDataStream's published layout (big-endian int32
precision, big-endian IEEE time and values) by byte-level comparison with a
numpy rendering, and by round trips through the context (GPU tests)."""
import os

import numpy as np
import pytest

import cases_def
import pyoracle
from drnum_b200 import _lib, cases
from drnum_b200._lib import DnError
from drnum_b200.api import CartesianPatch, PatchGrid
from test_overlap import TABLE_KEYS

needs_ref = pytest.mark.skipif(not pyoracle.ref_available(), reason="compiled reference (oracle/_ref) not built")

HAND_WRITTEN = """1001 // first patch, hand-written: tabs, commas, leading zeroes
{
\t0.25 0.5 -0.125
  1 0 0
  0 1 0
  2
  6 5 7
  0 2 0 2   0 0
  0.6 0.5 0.7
  fx fy  fz
  0007, 00 ; 12 0 0 03
  0
}
1001 comment of the second patch
{ 1.1 0.5 -0.125  1 0 0  0 1 0  2.0
  12 10 14   2 0 2 0 0 0   0.6 0.5 0.7  fx fy fz 0 0 0 0 0 0 0 }
0
trailing text after the end marker is not read
"""


def _layout_grid(layout, scale_io=1.0):
    grid = PatchGrid()
    for p in layout:
        grid.insertPatch(CartesianPatch(*p["n"], lengths=p["length"], origin=p["origin"],
                                        periodic=(False, False, False), seek=p["seek"]))
    return grid


def _compare_with_reference(path, scale, grid, codes):
    ref = pyoracle.RefGrid(None, 0, threads=1, grid_file=os.path.basename(path), scale=scale)
    try:
        assert ref.num_patches() == grid.getNumPatches()
        for i in range(grid.getNumPatches()):
            n, o, d, c = ref.patch_info(i)
            p = grid.getPatch(i)
            assert tuple(n) == (p.sizeI(), p.sizeJ(), p.sizeK())
            assert tuple(o) == p.origin, (i, o, p.origin)
            assert tuple(d) == (p.dx(), p.dy(), p.dz()), (i, d)
            assert c == codes[i], (i, c, codes[i])
        grid.computeDependencies()
        for i in range(grid.getNumPatches()):
            t = ref.tables(i)
            for k in TABLE_KEYS:
                assert np.array_equal(np.asarray(grid.tables[i][k]), t[k]), (i, k)
    finally:
        ref.close()


@needs_ref
def test_hand_written_grid_file_reads_as_the_reference(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    path = tmp_path / "hand.grid"
    path.write_text(HAND_WRITTEN)
    grid = PatchGrid()
    codes = grid.readGrid(str(path), scale=0.5)
    assert grid.getNumPatches() == 2
    assert grid.getPatch(0).seek == (0, 2, 0, 2, 0, 0)
    assert codes[0] == "fx fy fz 7 0 12 0 0 3 0"
    _compare_with_reference(str(path), 0.5, grid, codes)


@needs_ref
@pytest.mark.parametrize("name", ["random6", "octants_ragged", "embedded"])
def test_written_grid_file_reads_back_and_as_the_reference(tmp_path, monkeypatch, name):
    monkeypatch.chdir(tmp_path)
    layout = cases_def.grid_layout(name)
    src = _layout_grid(layout)
    path = tmp_path / f"{name}.grid"
    codes_in = [f"fx fy fz {q} 0 0 0 0 0 0" for q in range(len(layout))]
    src.writeGrid(str(path), codes_in)
    grid = PatchGrid()
    codes = grid.readGrid(str(path))
    assert codes == codes_in
    for a, b in zip(src.m_Patches, grid.m_Patches):
        assert a.desc().ni == b.desc().ni and a.seek == b.seek
        assert a.origin == b.origin and a.lengths == b.lengths
    _compare_with_reference(str(path), 1.0, grid, codes)


@pytest.mark.parametrize("text", [
    "1002 unknown type { 0 0 0 1 0 0 0 1 0 1 4 4 4 0 0 0 0 0 0 1 1 1 }\n0\n",
    "1001 rotated { 0 0 0 0 1 0 1 0 0 1 4 4 4 0 0 0 0 0 0 1 1 1 }\n0\n",
    "1001 short { 0 0 0 1 0 0 0 1 0 1 4 4 }\n0\n",
    "1001 unclosed { 0 0 0 1 0 0 0 1 0 1 4 4 4 0 0 0 0 0 0 1 1 1\n",
    "1001 no cells { 0 0 0 1 0 0 0 1 0 1 0 4 4 0 0 0 0 0 0 1 1 1 }\n0\n",
])
def test_malformed_grid_files_are_rejected(tmp_path, text):
    path = tmp_path / "bad.grid"
    path.write_text(text)
    with pytest.raises(DnError):
        PatchGrid().readGrid(str(path))


def test_missing_grid_file_is_an_error(tmp_path):
    with pytest.raises(DnError):
        PatchGrid().readGrid(str(tmp_path / "none.grid"))


def dnd_bytes(time, fields, prec=8):
    """QDataStream rendering of a .dnd file (big-endian)."""
    t = ">f8" if prec == 8 else ">f4"
    out = np.array([prec], ">i4").tobytes() + np.array([time], t).tobytes()
    for f in fields:
        out += np.ascontiguousarray(f, dtype=np.float64).astype(t).tobytes()
    return out


@pytest.mark.gpu
def test_dnd_write_matches_qdatastream_layout_and_reads_back(tmp_path):
    from drnum_b200.api import AusmPlus, B200CartesianIterator
    layout = cases_def.grid_layout("pair_x")
    it = B200CartesianIterator(AusmPlus(), 0, _lib.DN_FP64)
    states = cases.grid_state(layout)
    for p, U in zip(layout, states):
        cp = CartesianPatch(*p["n"], lengths=p["length"], origin=p["origin"], periodic=(False, False, False),
                            seek=p["seek"])
        cp.setField(0, U)
        it.addPatch(cp)
    it.updateDevice(fields=(0,))
    name = it.writeData(0, str(tmp_path / "step"), 0.125, 42)
    assert name.endswith("step_000042.dnd")
    raw = open(name, "rb").read()
    assert raw == dnd_bytes(0.125, states)
    # read into field 1 and compare; a precision-4 file is accepted too
    assert it.readData(1, str(tmp_path / "step_000042")) == 0.125
    it.updateHost(fields=(1,))
    for cp, U in zip(it.m_Patches, states):
        assert np.array_equal(cp.getField(1), U)
    f4 = tmp_path / "single.dnd"
    f4.write_bytes(dnd_bytes(2.5, states, prec=4))
    assert it.readData(2, str(f4)) == 2.5
    it.updateHost(fields=(2,))
    for cp, U in zip(it.m_Patches, states):
        assert np.array_equal(cp.getField(2), U.astype(np.float32).astype(np.float64))
    # a file for other patches is refused
    short = tmp_path / "short.dnd"
    short.write_bytes(dnd_bytes(1.0, states[:1]))
    with pytest.raises(DnError):
        it.readData(0, str(short))
    it.close()
