"""The regrid step on the device (fac_tag_gradient, fac_cluster_tags)
against the reference's own tagging and Berger-Rigoutsos clustering.

tests/golden/ref_br_<case>.npz hold the tags of the FAC_adaptive test's
AdaptivePoisson estimate and the boxes of mesh::BergerRigoutsos for the
cases of tests/br_cases.py (oracle/_ref/br_ref_driver).  The device tags
must equal them bit for bit and the boxes as a set; several problems in one
context are tagged and clustered each on its own and all at once
(fac_cluster_tags_all).
"""
import os

import numpy as np
import pytest

import br_cases
from samrai_b200 import fac
from oracle.oracle import U

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fixture(name):
    fx = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    tags = np.unpackbits(fx["tags_packed"])[:int(fx["ntags"][0])]
    return fx, tags


@pytest.mark.parametrize("name", list(br_cases.CASES))
def test_device_regrid_matches_reference(name, require_gpu):
    fx, want = _fixture(name)
    c = br_cases.CASES[name]
    p = br_cases.problem(name)
    g = fac.FacContext([p])
    g.upload(U, 0, 0, p.u0[0])
    cnt = g.tag_gradient(U, 0, c["threshold"])
    assert int(cnt[0]) == int(fx["tagged"][0])
    assert np.array_equal(g.download_tags(0, 0), want)
    boxes = g.cluster_tags(0, 0, br_cases.bound_boxes(name), c["min_box"], c["max_box"],
                           c["efficiency"], c["combine"])
    assert np.array_equal(br_cases.sorted_boxes(boxes), br_cases.sorted_boxes(fx["boxes"]))
    g.close()


def test_batched_problems_tag_and_cluster_each(require_gpu):
    names = ["br_3d", "br_3d_eff"]
    probs = [br_cases.problem(n) for n in names]
    g = fac.FacContext(probs)
    for i, p in enumerate(probs):
        g.upload(U, i, 0, p.u0[0])
    thr = br_cases.CASES[names[0]]["threshold"]
    cnt = g.tag_gradient(U, 0, thr)
    for i, n in enumerate(names):
        c = br_cases.CASES[n]
        fx, want = _fixture(n)
        if c["threshold"] == thr:
            assert int(cnt[i]) == int(fx["tagged"][0])
            assert np.array_equal(g.download_tags(i, 0), want)
    # per problem with its own threshold: retag and cluster
    for i, n in enumerate(names):
        c = br_cases.CASES[n]
        fx, want = _fixture(n)
        cnt = g.tag_gradient(U, 0, c["threshold"])
        assert int(cnt[i]) == int(fx["tagged"][0])
        boxes = g.cluster_tags(i, 0, br_cases.bound_boxes(n), c["min_box"], c["max_box"],
                               c["efficiency"], c["combine"])
        assert np.array_equal(br_cases.sorted_boxes(boxes), br_cases.sorted_boxes(fx["boxes"]))
    g.close()


def test_cluster_all_problems_at_once(require_gpu):
    """fac_cluster_tags_all over problems of different sizes and parameters
    sharing one threshold: the same boxes, in the same order, as
    fac_cluster_tags problem by problem, and the reference's boxes where the
    fixture's threshold is the one used."""
    names = ["br_3d", "br_3d_eff"]
    probs = [br_cases.problem(n) for n in names]
    g = fac.FacContext(probs)
    for i, p in enumerate(probs):
        g.upload(U, i, 0, p.u0[0])
    c0 = br_cases.CASES[names[0]]
    g.tag_gradient(U, 0, c0["threshold"])
    bounds = [br_cases.bound_boxes(n) for n in names]
    one = [g.cluster_tags(i, 0, bounds[i], c0["min_box"], c0["max_box"], c0["efficiency"],
                          c0["combine"]) for i in range(len(names))]
    allb = g.cluster_tags_all(0, bounds, c0["min_box"], c0["max_box"], c0["efficiency"],
                              c0["combine"])
    assert len(allb) == len(names)
    for a, b in zip(one, allb):
        assert np.array_equal(a, b)
    fx, _ = _fixture(names[0])
    assert np.array_equal(br_cases.sorted_boxes(allb[0]), br_cases.sorted_boxes(fx["boxes"]))
    g.close()
