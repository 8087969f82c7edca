"""The regrid step's CPU restatement (oracle/br_oracle.py) against the
reference's own tagging and Berger-Rigoutsos clustering.

tests/golden/ref_br_<case>.npz hold what SAMRAI itself computed for the
cases of tests/br_cases.py (oracle/_ref/br_ref_driver: the FAC_adaptive
test's AdaptivePoisson adaption estimate with its threshold test, and
mesh::BergerRigoutsos::findBoxesContainingTags), made by
tests/golden/make_br_fixtures.py.  The restatement must give the same tags
bit for bit and the same set of boxes.
"""
import os

import numpy as np
import pytest

import br_cases
from oracle import br_oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def oracle_tags(p, threshold):
    out = []
    for b, ug in zip(p.levels[0].boxes, br_cases.patch_arrays(p, p.u0[0], 1)):
        n = [b[3 + a] - b[a] + 1 for a in range(3)]
        shape = (n[2] + 2, n[1] + 2, n[0] + 2) if p.dim == 3 else (n[1] + 2, n[0] + 2)
        est = br_oracle.adaption_estimate(ug.reshape(shape), p.dim)
        out.append((est > threshold).astype(np.uint8).reshape(-1))
    return np.concatenate(out)


def dense_tags(p, tags):
    n = p.n0
    d = np.zeros((n[2], n[1], n[0]), dtype=np.int64)
    for b, t in zip(p.levels[0].boxes, br_cases.patch_arrays(p, tags, 0)):
        m = [b[3 + a] - b[a] + 1 for a in range(3)]
        d[b[2]:b[5] + 1, b[1]:b[4] + 1, b[0]:b[3] + 1] = t.reshape(m[2], m[1], m[0])
    return d if p.dim == 3 else d[0]


@pytest.mark.parametrize("name", list(br_cases.CASES))
def test_restatement_matches_reference_regrid(name):
    fx = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    c = br_cases.CASES[name]
    p = br_cases.problem(name)
    tags = oracle_tags(p, c["threshold"])
    want = np.unpackbits(fx["tags_packed"])[:int(fx["ntags"][0])]
    assert np.array_equal(tags, want)
    cl = br_oracle.Clusterer(dense_tags(p, tags), [0, 0, 0], p.dim, c["min_box"], c["max_box"],
                             c["efficiency"], c["combine"])
    boxes = cl.cluster(br_cases.bound_boxes(name))
    pad = [0] * (3 - p.dim)
    got = np.array([list(lo) + pad + list(hi) + pad for lo, hi in boxes], dtype=np.int64)
    assert np.array_equal(br_cases.sorted_boxes(got), br_cases.sorted_boxes(fx["boxes"]))
    # the boxes cover every tag and do not overlap
    cover = np.zeros_like(dense_tags(p, tags))
    for b in got.reshape(-1, 6):
        sl = tuple(slice(b[a], b[3 + a] + 1) for a in reversed(range(p.dim)))
        cover[sl] += 1
    assert cover.max() <= 1
    assert np.all(cover[dense_tags(p, tags) > 0] == 1)
