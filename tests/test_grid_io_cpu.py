"""grid.dat and xyz.dat: the library's reader against the reference's own
MG_Initial (init.c:313-440, compiled into oracle/_ref) on files in each of the three
formats the reference reads, and round trips through the library's writer.  Host code
only: no GPU."""
import os

import numpy as np
import pytest

import vfs_b200 as vfs
from vfs_b200 import cases
from oracle import ref

NAMES = {vfs.GRID_ASCII: "grid.dat", vfs.GRID_BINARY: "grid.dat", vfs.GRID_XYZ: "xyz.dat"}


def _case(fmt):
    # xyz.dat holds tensor-product grids only; the other formats take the curvilinear one
    return cases.channel(6, 5, 7, wavy=0.0 if fmt == vfs.GRID_XYZ else 0.1)


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("fmt", [vfs.GRID_ASCII, vfs.GRID_BINARY, vfs.GRID_XYZ])
def test_reader_matches_the_reference_reader(fmt):
    case = _case(fmt)
    name = NAMES[fmt]

    def writer(d):
        vfs.grid_write(os.path.join(d, name), case.X, case.Y, case.Z, fmt)

    flags = {"binary_input": int(fmt == vfs.GRID_BINARY), "xyz_input": int(fmt == vfs.GRID_XYZ)}
    try:
        R = ref.Reference(case, extra_globals=flags, grid_writer=writer)
        coor = R.get("coor")
        x, y, z = vfs.grid_read(os.path.join(R.dir, name), fmt)
        R.close()
    finally:
        ref.set_global("binary_input", 0)
        ref.set_global("xyz_input", 0)
    KM, JM, IM = x.shape
    assert (IM, JM, KM) == (case.IM, case.JM, case.KM)
    for c, a in enumerate((x, y, z)):
        np.testing.assert_array_equal(a, coor[:KM, :JM, :IM, c])
    for a, b in ((x, case.X), (y, case.Y), (z, case.Z)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("fmt", [vfs.GRID_ASCII, vfs.GRID_BINARY, vfs.GRID_XYZ])
def test_round_trip(fmt, tmp_path):
    case = _case(fmt)
    p = str(tmp_path / NAMES[fmt])
    vfs.grid_write(p, case.X, case.Y, case.Z, fmt)
    x, y, z = vfs.grid_read(p, fmt)
    for a, b in ((x, case.X), (y, case.Y), (z, case.Z)):
        np.testing.assert_array_equal(a, b)
    # the reference's scaling on reading: v / cl * L_dim
    xs, _, _ = vfs.grid_read(p, fmt, cl=2.0, L_dim=3.0)
    np.testing.assert_array_equal(xs, case.X / 2.0 * 3.0)


def test_second_block_of_a_two_block_ascii_file(tmp_path):
    """Blocks follow each other (header, x, y, z); the reader skips to the one asked for."""
    a, b = cases.channel(4, 3, 5), cases.channel(5, 4, 3, wavy=0.1)
    p = str(tmp_path / "grid.dat")
    with open(p, "w") as f:
        f.write("2\n")
        for c in (a, b):
            f.write("%d %d %d\n" % (c.IM, c.JM, c.KM))
            for arr in (c.X, c.Y, c.Z):
                np.savetxt(f, arr.reshape(-1), fmt="%.17e")
    x, y, z = vfs.grid_read(p, vfs.GRID_ASCII, block=1)
    for u, v in ((x, b.X), (y, b.Y), (z, b.Z)):
        np.testing.assert_array_equal(u, v)
    with pytest.raises(vfs.VfsError):
        vfs.grid_read(p, vfs.GRID_ASCII, block=2)


def test_errors(tmp_path):
    c = cases.channel(4, 3, 5, wavy=0.1)
    with pytest.raises(vfs.VfsError):   # xyz.dat cannot hold a curvilinear grid
        vfs.grid_write(str(tmp_path / "xyz.dat"), c.X, c.Y, c.Z, vfs.GRID_XYZ)
    with pytest.raises(vfs.VfsError):
        vfs.grid_read(str(tmp_path / "missing.dat"), vfs.GRID_ASCII)
    p = str(tmp_path / "grid.dat")
    vfs.grid_write(p, c.X, c.Y, c.Z, vfs.GRID_BINARY)
    with open(p, "r+b") as f:
        f.truncate(200)
    with pytest.raises(vfs.VfsError):
        vfs.grid_read(p, vfs.GRID_BINARY)
