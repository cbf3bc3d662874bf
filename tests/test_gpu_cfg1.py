"""Bit-exact parity at full size: the 1025 x 1025 wavy cloth (2,097,152
triangles, thickness 1e-4), both V1 draws of the timed step.

The first draw takes a full LBVH build; the second (same F, V1 redrawn) takes
the refit-only path.  For each, the device's candidate-stencil set, discrete-
pair set, hit set and hit -> toi map are compared with the reference's, as
order-independent digests (tests/digest.py) recorded from the reference build
by tests/golden/make_golden.py (cfg1_digests.json): candidates as filter_pair
saw them (BVHTree.cpp:345-395), hits as append_pair received them
(BVHTree.cpp:262), discrete pairs as append_discrete did (BVHTree.cpp:281),
and every hit's toi as the reference's NarrowPhaseACCD::query_ccd_* returns
it on the device's stencil orientation.  Equal digests over these sets mean
equal sets, with overwhelming probability."""
import hashlib
import json
import os

import numpy as np
import pytest

from digest import hit_rows, set_digest, set_rows
from mclccd_b200 import PREC_FP64, BVHTree, scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "cfg1_digests.json")


def check_draw(t, g):
    c = t.counts()
    assert (c["leaf_pairs"], c["vf"], c["ee"]) == (g["n_leaf_pairs"], g["n_vf"], g["n_ee"])
    cs, cv = t.candidates()
    assert set_digest(set_rows(cs, cv)) == g["candidates"]
    del cs, cv
    hs, hv, ht = t.hits()
    assert set_digest(set_rows(hs, hv)) == g["hits"]
    assert set_digest(hit_rows(hs, hv, ht)) == g["hit_toi"]
    del hs, hv, ht
    d = t.discrete()
    assert set_digest(np.sort(d, axis=1)) == g["discrete"]


def test_full_size_cloth_both_draws_against_reference_digests():
    with open(GOLD) as f:
        gold = json.load(f)
    V0, V1a, F, eta = scenes.wavy_cloth(1025, seed=0)
    V1b = scenes.wavy_redraw(V0, 1)
    assert hashlib.sha256(F.tobytes()).hexdigest() == gold["F_sha256"]
    assert hashlib.sha256(V0.tobytes()).hexdigest() == gold["V0_sha256"]
    assert hashlib.sha256(V1a.tobytes()).hexdigest() == gold["draws"]["a"]["V1_sha256"]
    assert hashlib.sha256(V1b.tobytes()).hexdigest() == gold["draws"]["b"]["V1_sha256"]
    t = BVHTree(3, precision=PREC_FP64)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1a, F)
    t.traverse(V0, V1a, F)
    check_draw(t, gold["draws"]["a"])
    # same F: the refit-only update (no new hierarchy build)
    assert t.build_stats() == (1, 0)
    t.update(V0, V1b, F)
    assert t.build_stats() == (1, 0)
    t.traverse(V0, V1b, F)
    check_draw(t, gold["draws"]["b"])
