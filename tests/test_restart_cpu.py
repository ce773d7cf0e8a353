"""Restart files: the library's PETSc-binary Vec reader and writer
against the reference's own Ucont_P_Binary_Output / Ucont_P_Binary_Input (main.c:765,
main.c:394), compiled into the oracle with the shim's binary viewer.  Host code only."""
import os
import tempfile

import numpy as np
import pytest

from oracle import ref
import vfs_b200 as vfs
from helpers import build_pair, small_channel

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _reference_with_state(les=False):
    case = small_channel(wavy=0.1)
    case.les = 2 if les else 0
    R = ref.Reference(case)
    rng = np.random.Generator(np.random.Philox(21))
    fields = {"Ucont": rng.standard_normal(R.shape + (3,)), "Ucat": rng.standard_normal(R.shape + (3,)),
              "P": rng.standard_normal(R.shape), "Nvert": np.zeros(R.shape)}
    fields["Nvert"][3:5, 2:4, 4:7] = 3.0
    R.set("Ucont", fields["Ucont"])
    R.set("Ucat", fields["Ucat"])
    R.set("P", fields["P"])
    R.set("Nvert", fields["Nvert"])
    if les:
        fields["Cs"] = rng.random(R.shape) * 0.1
        R.set("lCs", fields["Cs"])
    return case, R, fields


FILES = (("vfield", "Ucont"), ("ufield", "Ucat"), ("pfield", "P"), ("nvfield", "Nvert"))


@pytest.mark.parametrize("les", [False, True])
def test_reference_files_read_by_the_library(les):
    case, R, fields = _reference_with_state(les)
    with tempfile.TemporaryDirectory() as d:
        R.restart_output(d, 7)
        npts = int(np.prod(R.shape))
        for stem, name in FILES + ((("cs_", "Cs"),) if les else ()):
            path = os.path.join(d, "%s%06d_0.dat" % (stem, 7))
            a = fields[name]
            got = vfs.petsc_vec_read(path, a.size)
            np.testing.assert_array_equal(got, a.reshape(-1), err_msg=stem)
            assert os.path.getsize(path) == 8 + 8 * a.size
        with pytest.raises(vfs.VfsError):
            vfs.petsc_vec_read(os.path.join(d, "pfield%06d_0.dat" % 7), npts + 1)
    R.close()


@pytest.mark.parametrize("les", [False, True])
def test_library_files_read_by_the_reference(les):
    case, R, fields = _reference_with_state(les)
    with tempfile.TemporaryDirectory() as d:
        R.restart_output(d, 3)                      # the reference's own files, for bytes
        e = os.path.join(d, "ours")
        os.mkdir(e)
        for stem, name in FILES + ((("cs_", "Cs"),) if les else ()):
            vfs.petsc_vec_write(os.path.join(e, "%s%06d_0.dat" % (stem, 3)), fields[name])
            with open(os.path.join(d, "%s%06d_0.dat" % (stem, 3)), "rb") as f1, \
                    open(os.path.join(e, "%s%06d_0.dat" % (stem, 3)), "rb") as f2:
                assert f1.read() == f2.read(), stem
        R2 = ref.Reference(case)
        R2.restart_input(e, 3)
        np.testing.assert_array_equal(R2.get("Ucont"), fields["Ucont"])
        np.testing.assert_array_equal(R2.get("lUcont"), fields["Ucont"])
        np.testing.assert_array_equal(R2.get("Ucont_o"), fields["Ucont"])
        np.testing.assert_array_equal(R2.get("Ucat"), fields["Ucat"])
        np.testing.assert_array_equal(R2.get("lUcat_old"), fields["Ucat"])
        np.testing.assert_array_equal(R2.get("P"), fields["P"])
        np.testing.assert_array_equal(R2.get("lP"), fields["P"])
        if les:
            np.testing.assert_array_equal(R2.get("lCs"), fields["Cs"])
        R2.close()
    R.close()
