"""Generate the golden known-answer fixtures from the reference's own tests.

The reference test script (test_fof.py) builds its known-answer inputs with
``generate_predictable_halo`` (test_fof.py:361-458) under fixed legacy
``np.random`` seeds and asserts exact answers (test_fof.py:653-969,
1022-1169).  That script imports matplotlib at module level, so it cannot be
imported here; this generator parses it, executes only the generator
function, replays each test's random draws in the test's own order, and
stores inputs plus the test's expected answers as ``.npz`` fixtures in this
directory.

Usage (needs the reference checkout, read-only):
    python tests/golden/make_golden.py path/to/reference   (or PYFOF_REFERENCE=...)
The fixtures are committed; tests never read the reference tree.
"""
from __future__ import annotations

import ast
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LINK = 2.0          # LINKING_LENGTH, test_fof.py:20
NP_MIN = 10         # NP_HALO_MIN, test_fof.py:21
L_BOX = 512.0       # L_BOX, test_fof.py:19
SHIFTS = [np.array([-50.0, -50.0, 0.0]), np.array([50.0, -50.0, 0.0]),
          np.array([0.0, 50.0, 30.0])]   # test_fof.py:821-825 and :890-894


def load_generator(ref_root: str):
    src_path = os.path.join(ref_root, "test_fof.py")
    src = open(src_path, encoding="utf-8").read()
    tree = ast.parse(src)
    fn = next(n for n in tree.body
              if isinstance(n, ast.FunctionDef) and n.name == "generate_predictable_halo")
    mod = ast.Module(body=[fn], type_ignores=[])
    ns = {"np": np}
    exec(compile(mod, src_path, "exec"), ns)
    return ns["generate_predictable_halo"]


def main(ref_root: str) -> None:
    gen = load_generator(ref_root)
    out = {}

    # test_predictable_halo (test_fof.py:653-729)
    np.random.seed(999)
    xp, exp, _, _ = gen(n_halo_particles=200, linking_length=LINK, n_noise_particles=400, seed=999)
    out["predictable_halo"] = dict(xp=xp, expected=exp)

    # test_predictable_halo_with_velocity (test_fof.py:734-799)
    np.random.seed(888)
    xp, exp, _, _ = gen(n_halo_particles=200, linking_length=LINK, n_noise_particles=400, seed=888)
    vp = np.random.randn(3, 600).astype(np.float64) * 0.1
    n_high = max(1, int(200 * 0.1))
    hidx = np.where(exp)[0]
    high = np.random.choice(hidx, n_high, replace=False)
    vp[:, high] *= 100.0
    out["predictable_halo_velocity"] = dict(xp=xp, vp=vp, expected=exp, high_v=high,
                                            expected_bound=np.int64(200 - n_high))

    # test_multiple_predictable_halos (test_fof.py:804-866)
    np.random.seed(777)
    xs, es = [], []
    for i in range(3):
        xp, exp, _, _ = gen(n_halo_particles=100, linking_length=LINK, n_noise_particles=200,
                            seed=777 + i)
        xs.append(xp + SHIFTS[i].reshape(3, 1))
        es.append(exp)
    out["multiple_halos"] = dict(xp0=xs[0], xp1=xs[1], xp2=xs[2], expected=np.hstack(es))

    # test_multiple_predictable_halos_with_velocity (test_fof.py:871-969)
    np.random.seed(666)
    xs, vs, es, hs = [], [], [], []
    for i in range(3):
        xp, exp, _, _ = gen(n_halo_particles=100, linking_length=LINK, n_noise_particles=200,
                            seed=666 + i)
        xp = xp + SHIFTS[i].reshape(3, 1)
        vp = np.random.randn(3, 300).astype(np.float64) * 0.1
        n_high = max(1, int(100 * 0.1))
        hidx = np.where(exp)[0]
        high = np.random.choice(hidx, n_high, replace=False)
        vp[:, high] *= 100.0
        xs.append(xp); vs.append(vp); es.append(exp); hs.append(high + 300 * i)
    out["multiple_halos_velocity"] = dict(
        xp0=xs[0], xp1=xs[1], xp2=xs[2], vp0=vs[0], vp1=vs[1], vp2=vs[2],
        expected=np.hstack(es), high_v=np.hstack(hs), expected_bound=np.int64(300 - 30))

    # test_new_features [1]-[4] (test_fof.py:1036-1149)
    np.random.seed(101)
    xs, vs = [], []
    for i in range(3):
        xp, _, _, _ = gen(100, LINK, 50, seed=101 + i)
        xs.append(xp + np.array([i * 100.0, 0.0, 0.0]).reshape(3, 1))
        vs.append(np.random.randn(3, 150).astype(np.float64) * 0.05)
    np.random.seed(202)
    xs1, _, _, _ = gen(100, LINK, 0, seed=202)
    vs1 = np.random.randn(3, 100).astype(np.float64) * 0.25
    out["new_features"] = dict(xp0=xs[0], xp1=xs[1], xp2=xs[2], vp0=vs[0], vp1=vs[1],
                               vp2=vs[2], nhalo_expected=np.int64(3), xp_single=xs1,
                               vp_single=vs1)

    # test_new_features [5] span guard input (test_fof.py:1155-1160)
    x = np.linspace(10.0, 35.0, 1050, endpoint=True)
    out["overspan"] = dict(xp=np.vstack([x, np.zeros(1050), np.zeros(1050)]),
                           vp=np.zeros((3, 1050)))

    for name, arrs in out.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrs)
        print("wrote", name, {k: getattr(v, "shape", v) for k, v in arrs.items()})


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYFOF_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set PYFOF_REFERENCE)")
    main(ref)
