"""Generate tests/golden/ref_br_<case>.npz: the reference's own tagging
(AdaptivePoisson's adaption estimate > threshold) and Berger-Rigoutsos
clustering (mesh::BergerRigoutsos::findBoxesContainingTags) of the cases in
tests/br_cases.py, run by oracle/_ref/br_ref_driver (built by
oracle/ref/build_ref.py from the reference's sources).

    python oracle/ref/build_ref.py
    python tests/golden/make_br_fixtures.py [case ...]

Each fixture holds the tags (ghost-0 arrays of the patches, packed bits),
their count, and the boxes in the order of the reference's new BoxLevel.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.ref import refio  # noqa: E402
import br_cases  # noqa: E402


def main(names):
    for name in names or list(br_cases.CASES):
        c = br_cases.CASES[name]
        p = br_cases.problem(name)
        out = refio.run_br(p, c["threshold"], br_cases.bound_boxes(name), c["min_box"],
                           c["max_box"], c["efficiency"], c["combine"])
        tags = out["tags"].astype(np.uint8)
        boxes = out["boxes"].reshape(-1, 6)
        path = os.path.join(HERE, f"ref_{name}.npz")
        np.savez_compressed(path, tags_packed=np.packbits(tags), ntags=np.array([tags.size]),
                            tagged=np.array([int(tags.sum())]), boxes=boxes,
                            seconds=out["seconds"])
        print(f"{name}: {int(tags.sum())} of {tags.size} cells tagged, {len(boxes)} boxes "
              f"-> {os.path.basename(path)}", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
