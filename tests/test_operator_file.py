"""The operator file (the reference's .dat layout: fmm_scale_invariant.h:86-160, fmm.h:83-153) read and
written by xfmm_precompute, against the reference's own files and the reference reading ours.

  * a file the reference wrote is loaded (not recomputed: the file is left as it was) and the FP64 path
    then agrees with the reference's output far more closely than with its own operators;
  * a file this library wrote is loaded by the reference (left unchanged by it), whose results with our
    operators agree with its results with its own within the FP64 tolerance;
  * a file of another configuration (other r0) is replaced, as the reference replaces it."""
import os

import numpy as np
import pytest

from oracle import orc, ref
from tests.golden_cases import load

pytestmark = pytest.mark.gpu

CASES = ["laplace_cube_p4", "yukawa_sphere_p4", "helmholtz_cube_p4"]


def _mod(kernel):
    import exafmm.helmholtz
    import exafmm.laplace
    import exafmm.modified_helmholtz
    return {"laplace": exafmm.laplace, "helmholtz": exafmm.helmholtz,
            "modified_helmholtz": exafmm.modified_helmholtz}[kernel]


def _ours(g, precision, filename):
    m = _mod(g["kernel"])
    if g["kernel"] == "laplace":
        fmm = m.LaplaceFmm(g["p"], g["ncrit"], filename=filename, precision=precision)
    elif g["kernel"] == "helmholtz":
        fmm = m.HelmholtzFmm(g["p"], g["ncrit"], g["wavek"], filename=filename, precision=precision)
    else:
        fmm = m.ModifiedHelmholtzFmm(g["p"], g["ncrit"], g["wavek"].real, filename=filename, precision=precision)
    tree = m.setup(m.init_sources(g["src"], g["q"]), m.init_targets(g["trg"]), fmm)
    return m.evaluate(tree, fmm)


def _reference(g, datdir):
    if not ref.available():
        pytest.skip("reference build oracle/_ref missing (make -C oracle ref)")
    f = ref.RefFmm(g["kernel"], g["p"], g["ncrit"], wavek=g["wavek"], datdir=str(datdir))
    f.setup(g["src"], g["q"], g["trg"])
    out = f.evaluate()
    path = f.datfile.decode()
    f.close()
    return out, path


def _bytes(path):
    with open(path, "rb") as fh:
        return fh.read()


@pytest.mark.parametrize("name", CASES)
def test_reference_file_is_read(tmp_path, name):
    g = load(name)
    ref_out, path = _reference(g, tmp_path)
    before = _bytes(path)
    out = _ours(g, "fp64", path)
    assert _bytes(path) == before  # read, not rewritten
    pe, ge = orc.rel_l2(out, ref_out)
    assert pe < 1e-12 and ge < 1e-12, (pe, ge)
    out_m = _ours(g, "mixed", path)  # the mixed path derives its operators from the same file
    pe, ge = orc.rel_l2(out_m, ref_out)
    assert pe < 5e-6 and ge < 5e-6, (pe, ge)


@pytest.mark.parametrize("name", CASES)
def test_written_file_is_read_by_the_reference(tmp_path, name):
    g = load(name)
    (tmp_path / "own").mkdir()
    own_out, ref_path = _reference(g, tmp_path / "own")
    ours_dir = tmp_path / "ours"
    ours_dir.mkdir()
    path = str(ours_dir / os.path.basename(ref_path))
    out = _ours(g, "fp64", path)  # computed here, file written in the reference's layout
    assert os.path.getsize(path) == os.path.getsize(ref_path)
    written = _bytes(path)
    ref_out, _ = _reference(g, ours_dir)  # the reference finds our file under its own name
    assert _bytes(path) == written  # loaded by the reference, not recomputed
    for a, b, tol in ((ref_out, own_out, 1e-9), (out, ref_out, 1e-12)):
        pe, ge = orc.rel_l2(a, b)
        assert pe < tol and ge < tol, (pe, ge, tol)


def test_file_of_another_configuration_is_replaced(tmp_path):
    g = load("laplace_cube_p4")
    path = str(tmp_path / "laplace_p4.dat")
    _ours(g, "fp64", path)
    first = _bytes(path)
    g2 = dict(g)
    g2["src"] = g["src"] * 2.0  # another bounding box: another r0
    g2["trg"] = g["trg"] * 2.0
    out = _ours(g2, "fp64", path)
    assert _bytes(path) != first  # replaced
    ex = orc.direct("laplace", g2["src"], g2["q"], g2["trg"][:200])
    pe, ge = orc.rel_l2(out[:200], ex)
    assert pe < 1e-2 and ge < 1e-2, (pe, ge)
