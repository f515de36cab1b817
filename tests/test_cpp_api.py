"""The exafmm-t C++ API (include/exafmm_t_b200.h) with a caller shaped like the reference's C++ drivers
(tests/fmm_laplace.cpp: get_bounds, build_tree, balance_tree, init_rel_coord, set_colleagues,
build_list, precompute, M2L_setup, upward_pass, downward_pass, verify), compiled with g++ against the
header and linked with libexafmm_b200.so.  On the GPU its results are compared with fixtures the
reference itself produced: tree geometry and leaf keys exactly, FP64 values within 1e-9 relative L2."""
import os
import struct
import subprocess

import numpy as np
import pytest

from oracle import orc
from tests.golden_cases import load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "fmm_drop_in.cpp")
LIBDIR = os.path.join(ROOT, "exafmm-t_b200")
KERNELS = {"laplace": 0, "modified_helmholtz": 1, "helmholtz": 2}


def _compile(tmp, nonadaptive):
    exe = os.path.join(str(tmp), "fmm_drop_in%s" % ("_na" if nonadaptive else ""))
    cmd = ["g++", "-std=c++14", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-o", exe, SRC, "-L", LIBDIR, "-lexafmm_b200", "-Wl,-rpath," + LIBDIR]
    if nonadaptive:
        cmd.insert(1, "-DNON_ADAPTIVE=1")
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


@pytest.mark.skipif(not os.path.exists(os.path.join(LIBDIR, "libexafmm_b200.so")), reason="library not built")
@pytest.mark.parametrize("nonadaptive", [False, True])
def test_header_compiles_and_links(tmp_path, nonadaptive):
    assert os.path.exists(_compile(tmp_path, nonadaptive))


def _run(exe, g, tmp, precision):
    kern = KERNELS[g["kernel"]]
    src, trg = g["src"], g["trg"]
    q = g["q"]
    qv = np.stack([q.real, q.imag], axis=1).ravel() if kern == 2 else np.asarray(q, np.float64)
    depth = g["depth_arg"] if g["depth_arg"] >= 0 else 0
    inp, outp = os.path.join(str(tmp), "in.bin"), os.path.join(str(tmp), "out.bin")
    with open(inp, "wb") as f:
        f.write(struct.pack("<5i", kern, g["p"], g["ncrit"], depth, precision))
        f.write(struct.pack("<2q", len(src), len(trg)))
        f.write(struct.pack("<2d", g["wavek"].real, g["wavek"].imag))
        for a in (src, qv, trg):
            f.write(np.ascontiguousarray(a, np.float64).tobytes())
    run = subprocess.run([exe, inp, outp], capture_output=True, text=True)
    assert run.returncode == 0, run.stderr
    raw = open(outp, "rb").read()
    depth_o, nl, nnl = struct.unpack_from("<3i", raw, 0)
    geo = np.frombuffer(raw, np.float64, 6, 12)
    keys = np.frombuffer(raw, np.uint64, nl, 12 + 48)
    vals = np.frombuffer(raw, np.float64, offset=12 + 48 + 8 * nl)
    vals = vals.reshape(len(trg), 4, 2) if kern == 2 else vals.reshape(len(trg), 4)
    if kern == 2:
        vals = vals[..., 0] + 1j * vals[..., 1]
    return dict(depth=depth_o, nleafs=nl, nnonleafs=nnl, x0=geo[:3], r0=geo[3], err=geo[4:6], keys=keys, out=vals)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["laplace_cube_p4", "laplace_plummer_p4", "laplace_uniform_p4",
                                  "yukawa_sphere_p4", "helmholtz_cube_p4"])
def test_reference_style_caller_matches_the_reference(tmp_path, name):
    g = load(name)
    exe = _compile(tmp_path, g["depth_arg"] >= 0)
    r = _run(exe, g, tmp_path, 0)
    t = g["tree"]
    assert r["depth"] == t["depth"] and r["r0"] == t["r0"]
    assert r["nleafs"] == len(t["leafs"]) and r["nnonleafs"] == len(t["nonleafs"])
    assert np.array_equal(r["keys"], t["key"][t["leafs"]])
    pe, ge = orc.rel_l2(r["out"], g["out"])
    assert pe < 1e-9 and ge < 1e-9, (pe, ge)
    assert np.all(np.isfinite(r["err"])) and r["err"][0] < 1e-2  # verify: FP64 direct sums, every target


@pytest.mark.gpu
def test_reference_style_caller_mixed_precision(tmp_path):
    g = load("laplace_cube_p4")
    r = _run(_compile(tmp_path, False), g, tmp_path, 1)
    pe, ge = orc.rel_l2(r["out"], g["out"])
    assert pe < 5e-6 and ge < 5e-6, (pe, ge)
