"""Generate tests/golden/ref_<case>.npz: full FAC solves by the reference's
own solver (oracle/_ref/fac_ref_driver, built by oracle/ref/build_ref.py
from the reference's sources) of the problems in tests/ref_cases.py.

    python oracle/ref/build_ref.py
    python tests/golden/make_ref_fixtures.py [case ...]

Each fixture holds the iteration count, convergence flag, final residual
norm, the composite residual norm after every cycle, the convergence
factors and, per level, SHA-256 digests of the solution (interior, and with
its ghost cells), a fingerprint, every SAMPLE-th value and, for the small
2-D cases, the whole array.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.ref import refio  # noqa: E402
import ref_cases  # noqa: E402


def main(names):
    for name in names or list(ref_cases.CASES):
        build, params, bc, full = ref_cases.CASES[name]
        prob = build()
        t = time.perf_counter()
        out = refio.run_reference(prob, params, bc)
        dt = time.perf_counter() - t
        rec = {k: out[k] for k in ("converged", "iterations", "residual", "hist", "factors")}
        for ln in range(prob.nlev):
            u = out[f"u{ln}"]
            m = ref_cases.interior_mask(prob, ln)
            rec[f"u{ln}_sha_interior"] = ref_cases.digest(u[m])
            rec[f"u{ln}_sha_all"] = ref_cases.digest(u)
            rec[f"u{ln}_summary"] = ref_cases.summarize(u)
            rec[f"u{ln}_sample"] = u[::ref_cases.SAMPLE]
            if full:
                rec[f"u{ln}"] = u
        path = os.path.join(HERE, f"ref_{name}.npz")
        np.savez_compressed(path, **rec)
        print(f"{name}: {int(out['iterations'][0])} cycles, converged {int(out['converged'][0])}, "
              f"residual {out['residual'][0]:.3e}, {dt:.1f} s -> {os.path.basename(path)}",
              flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
