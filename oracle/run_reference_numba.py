"""Time the reference's own numba CPU path (pykifmm2d/class_fmm.py's FMM) on
this host, as a second CPU baseline beside the oracle port.

TEST / MEASUREMENT INFRASTRUCTURE ONLY: bench.py's CPU-baseline leg runs this
file in a subprocess (NUMBA_NUM_THREADS must be set before numba loads).  The
product never imports it.

The reference comes from baseline/_ref (the unmodified package installed by
pip from the reference checkout).  It does not import on current numba as
shipped: its explicit signatures use the fixed-size array type i8[4]
(tree.py:14,38,71,86), so a temporary copy gets i8[4] -> i8[:]; no arithmetic
changes.  A fresh FMM object per run (a second build_expansions on one object
accumulates into stale check potentials, tree.py:414 with class_fmm.py:71).

Usage: python run_reference_numba.py <npz with x, y, tau> <nequiv> <ncutoff> <repeats>
Prints one JSON line: seconds per run (median), threads, numba version.
"""
import json
import os
import shutil
import statistics
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "baseline", "_ref", "pykifmm2d")


def shimmed():
    tmp = tempfile.mkdtemp(prefix="kifmm_refnb_")
    dst = os.path.join(tmp, "pykifmm2d")
    shutil.copytree(REF, dst, ignore=shutil.ignore_patterns("*.pyc", "__pycache__"))
    tp = os.path.join(dst, "tree.py")
    src = open(tp).read()
    open(tp, "w").write(src.replace("i8[4]", "i8[:]"))
    sys.path.insert(0, tmp)
    import pykifmm2d.class_fmm as C  # noqa: E402
    return C


def main():
    path, neq, cut, reps = sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4])
    import numba
    C = shimmed()

    @numba.njit("f8(f8,f8,f8,f8)", fastmath=True)
    def laplace_eval(sx, sy, tx, ty):
        return -0.25 / np.pi * np.log((tx - sx) ** 2 + (ty - sy) ** 2)

    kf = C.Get_Kernel_Functions(laplace_eval)
    nf = C.prepare_numba_functions_on_the_fly(laplace_eval)

    def run(x, y, tau):
        f = C.FMM(x, y, kf, nf, neq, cut)
        f.build_tree()
        f.precompute()
        f.build_expansions(tau)
        return f.evaluate_to_points(x, y, True)

    rng = np.random.default_rng(0)  # JIT warm-up on 5,000 points
    run(rng.uniform(-1, 1, 5000), rng.uniform(-1, 1, 5000), rng.standard_normal(5000))
    d = np.load(path)
    x, y, tau = d["x"], d["y"], d["tau"]
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        run(x, y, tau)
        ts.append(time.perf_counter() - t0)
    print(json.dumps({"seconds": statistics.median(ts), "runs": ts, "threads": numba.get_num_threads(),
                      "numba": numba.__version__, "n": int(x.size)}))


if __name__ == "__main__":
    main()
