"""Record files exchanged with oracle/_ref/fac_ref_driver, and a runner.

Record: int32 name length, name, int32 type (0 f64, 1 i32), int64 count,
values.  TEST INFRASTRUCTURE ONLY.
"""
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(os.path.dirname(HERE), "_ref", "fac_ref_driver")
BR_DRIVER = os.path.join(os.path.dirname(HERE), "_ref", "br_ref_driver")


def write(path, recs):
    with open(path, "wb") as fh:
        for name, arr in recs:
            a = np.asarray(arr)
            if a.dtype.kind in "iu":
                a, t = np.ascontiguousarray(a, dtype=np.int32), 1
            else:
                a, t = np.ascontiguousarray(a, dtype=np.float64), 0
            nb = name.encode()
            fh.write(struct.pack("<i", len(nb)) + nb + struct.pack("<iq", t, a.size))
            fh.write(a.tobytes())


def read(path):
    out = {}
    with open(path, "rb") as fh:
        data = fh.read()
    k = 0
    while k < len(data):
        (n,) = struct.unpack_from("<i", data, k)
        k += 4
        name = data[k:k + n].decode()
        k += n
        t, cnt = struct.unpack_from("<iq", data, k)
        k += 12
        dt = np.float64 if t == 0 else np.int32
        nb = cnt * (8 if t == 0 else 4)
        out[name] = np.frombuffer(data[k:k + nb], dtype=dt).copy()
        k += nb
    return out


def problem_records(prob, params, bc=None):
    """Input records of fac_ref_driver for a samrai_b200.configs.Problem;
    bc "faces" selects the driver's position-dependent Robin object."""
    boxes = np.concatenate([lv.boxes for lv in prob.levels]).astype(np.int32)
    recs = [("dim", [prob.dim]), ("nlev", [prob.nlev]),
            ("n0", np.array(list(prob.n0) + [1] * (3 - len(prob.n0)), dtype=np.int32)),
            ("ratio", np.array([lv.ratio for lv in prob.levels], dtype=np.int32).reshape(-1)),
            ("npatch", np.array([len(lv.boxes) for lv in prob.levels], dtype=np.int32)),
            ("boxes", boxes.reshape(-1)),
            ("xlo", np.array(list(prob.xlo) + [0.0] * (3 - len(prob.xlo)))),
            ("xup", np.array(list(prob.xup) + [1.0] * (3 - len(prob.xup)))),
            ("poisson", [float(prob.d_variable), prob.d_const, float(prob.c_kind), prob.c_const]),
            ("params", [params["max_cycles"], params["residual_tol"],
                        params["relative_residual_tol"], params["pre_sweeps"],
                        params["post_sweeps"], params["coarse_tol"], params["coarse_max_it"]])]
    if isinstance(bc, str) and bc == "faces":
        recs.append(("bc_faces", np.array([1], dtype=np.int32)))
    elif bc is not None:
        # Robin a u + b du/dn = g per side; without it the solver's own
        # Dirichlet path, boundary values from u0's ghost cells
        recs.append(("bc", np.concatenate([np.asarray(x, dtype=np.float64) for x in bc])))
    from samrai_b200 import configs
    for ln in range(prob.nlev):
        recs.append((f"f{ln}", prob.f[ln]))
        recs.append((f"u0{ln}", prob.u0[ln] if prob.u0 else
                     np.zeros(configs.field_size(prob, ln, 1))))
        if prob.d_variable:
            recs.append((f"d{ln}", prob.d[ln]))
        if prob.c_kind == 2:
            recs.append((f"c{ln}", prob.c[ln]))
    return recs


def available(driver=DRIVER):
    return os.access(driver, os.X_OK)


def run_reference(prob, params, bc=None, driver=DRIVER, timeout=3600, solution=True):
    """Solve `prob` with the reference's CellPoissonFACSolver; returns the
    driver's output records (without the solution arrays when `solution`
    is false)."""
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        recs = problem_records(prob, params, bc)
        if not solution:
            recs.append(("skip_u", np.array([1], dtype=np.int32)))
        write(fin, recs)
        r = subprocess.run([driver, fin, fout], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"fac_ref_driver failed ({r.returncode}): {r.stderr[-2000:]}")
        return read(fout)


def run_br(prob, threshold, bound, min_box, max_box, efficiency, combine, driver=BR_DRIVER,
           timeout=600):
    """Tag level 0 of `prob` (u from prob.u0[0]) by the reference's
    AdaptivePoisson estimate and cluster the tags with its BergerRigoutsos
    (oracle/_ref/br_ref_driver); returns the driver's records (tags, boxes,
    seconds)."""
    dim = prob.dim
    pad = [1] * (3 - dim)
    recs = [("dim", [dim]),
            ("n0", np.array(list(prob.n0[:dim]) + pad, dtype=np.int32)),
            ("boxes", np.asarray(prob.levels[0].boxes, dtype=np.int32).reshape(-1)),
            ("xlo", np.array(list(prob.xlo[:dim]) + [0.0] * (3 - dim))),
            ("xup", np.array(list(prob.xup[:dim]) + [1.0] * (3 - dim))),
            ("u", prob.u0[0]), ("threshold", [float(threshold)]),
            ("bound", np.asarray(bound, dtype=np.int32).reshape(-1)),
            ("min_box", np.array(list(min_box[:dim]) + pad, dtype=np.int32)),
            ("max_box", np.array(list(max_box[:dim]) + [0] * (3 - dim), dtype=np.int32)),
            ("efficiency", [float(efficiency)]), ("combine", [float(combine)])]
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        write(fin, recs)
        r = subprocess.run([driver, fin, fout], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"br_ref_driver failed ({r.returncode}): {r.stderr[-2000:]}")
        return read(fout)
