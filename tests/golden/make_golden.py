"""Generate the golden fixtures in tests/golden/ from the REFERENCE itself.

Runs the unmodified exafmm-t headers (built into oracle/_ref by oracle/Makefile)
on small seeded inputs and stores inputs, tree/list dumps and potentials+gradients
as compressed .npz files.  Needs the reference sources (to build oracle/_ref), so
it runs in the development container only; the fixtures it writes are committed.

    python tests/golden/make_golden.py         # every fixture
    python tests/golden/make_golden.py f32     # only the single-precision reference fixtures
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import ref  # noqa: E402


def points(kind, n, rng):
    if kind == "cube":
        return rng.random((n, 3))
    if kind == "sphere":
        g = rng.normal(size=(n, 3))
        return g / np.linalg.norm(g, axis=1)[:, None]
    if kind == "plummer":
        x = rng.random(n)
        r = np.minimum(1.0 / np.sqrt(x ** (-2.0 / 3.0) - 1.0), 10.0)
        u = rng.normal(size=(n, 3))
        return u / np.linalg.norm(u, axis=1)[:, None] * r[:, None]
    raise ValueError(kind)


CASES = [
    # name, kernel, wavek, p, ncrit, dist, nsrc, ntrg (0 = same as sources), nonadaptive depth
    ("laplace_cube_p4", "laplace", 0.0, 4, 32, "cube", 2000, 0, None),
    ("laplace_cube_p6_targets", "laplace", 0.0, 6, 64, "cube", 3000, 1500, None),
    ("laplace_plummer_p4", "laplace", 0.0, 4, 16, "plummer", 3000, 0, None),
    ("laplace_uniform_p4", "laplace", 0.0, 4, 32, "cube", 2000, 0, 3),
    ("yukawa_sphere_p4", "modified_helmholtz", 10.0, 4, 32, "sphere", 2000, 0, None),
    ("helmholtz_cube_p4", "helmholtz", 5.0 + 0.0j, 4, 32, "cube", 1500, 0, None),
]


# the reference's single-precision build (-DFLOAT) next to its FP64 build and FP64 direct sums at
# every target: pins the mixed path against the reference's own FP32 FMM
CASES_F32 = [
    # name, kernel, wavek, p, ncrit, dist, n
    ("f32ref_laplace_cube_p8", "laplace", 0.0, 8, 32, "cube", 8000),
    ("f32ref_yukawa_sphere_p6", "modified_helmholtz", 10.0, 6, 32, "sphere", 5000),
]


def main_f32():
    from oracle import orc
    for i, (name, kern, k, p, ncrit, dist, n) in enumerate(CASES_F32):
        rng = np.random.default_rng(200 + i)
        x = points(dist, n, rng)
        q = rng.uniform(-1, 1, n)
        outs = {}
        for tag, fp32 in (("out32", True), ("out64", False)):
            f = ref.RefFmm(kern, p, ncrit, wavek=k, fp32=fp32)
            f.setup(x, q, x)
            outs[tag] = f.evaluate()
            f.close()
        # FP64 direct sums at every target (an error sampled on a subset can miss where the FP32 build
        # is worst)
        direct = orc.direct(kern, x, q, x, k) if kern != "laplace" else orc.direct(kern, x, q, x)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), kernel=kern, wavek=complex(k), p=p, ncrit=ncrit,
                            src=x, q=q, direct=direct, **outs)
        print(name, "f32 vs direct", orc.rel_l2(outs["out32"], direct), "bytes",
              os.path.getsize(os.path.join(HERE, name + ".npz")))


def main():
    for i, (name, kern, k, p, ncrit, dist, ns, nt, depth) in enumerate(CASES):
        rng = np.random.default_rng(100 + i)
        src = points(dist, ns, rng)
        trg = src if nt == 0 else points(dist, nt, rng)
        if kern == "helmholtz":
            q = rng.uniform(-1, 1, ns) + 1j * rng.uniform(-1, 1, ns)
        else:
            q = rng.uniform(-1, 1, ns)
        f = ref.RefFmm(kern, p, ncrit, wavek=k, nonadaptive_depth=depth)
        f.setup(src, q, trg)
        out = f.evaluate()
        d = f.dump()
        f.close()
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), kernel=kern, wavek=complex(k), p=p, ncrit=ncrit,
            depth_arg=-1 if depth is None else depth, src=src, trg=trg, q=q, out=out,
            **{"tree_" + key: v for key, v in d.items() if isinstance(v, np.ndarray)},
            tree_depth=d["depth"], tree_r0=d["r0"])
        print(name, "nodes", len(d["key"]), "depth", d["depth"], "bytes",
              os.path.getsize(os.path.join(HERE, name + ".npz")))
    # P2P kernels: reference SIMD gradient_P2P (laplace.h:91-164 and twins)
    rng = np.random.default_rng(7)
    s = rng.random((257, 3))
    t = np.concatenate([rng.random((190, 3)), s[:10]])  # includes coincident points (r == 0 skipped)
    q = rng.uniform(-1, 1, 257)
    qc = q + 1j * rng.uniform(-1, 1, 257)
    np.savez_compressed(
        os.path.join(HERE, "p2p_kernels.npz"), src=s, trg=t, q=q, qc=qc,
        laplace=ref.gradient_p2p("laplace", s, q, t),
        modified_helmholtz=ref.gradient_p2p("modified_helmholtz", s, q, t, 10.0),
        helmholtz=ref.gradient_p2p("helmholtz", s, qc, t, 5.0 + 10.0j))
    print("p2p_kernels written")


if __name__ == "__main__":
    if sys.argv[1:] == ["f32"]:
        main_f32()
    else:
        main()
        main_f32()
