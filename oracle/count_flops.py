"""FP64 flops per stencil of the narrow phase, counted on the oracle.

TEST / MEASUREMENT INFRASTRUCTURE: runs oracle/flops.cpp (the oracle's
distance routines on a counting number type) over the candidate stencils of
a workload and prints the flops per VF and per EE stencil, for the
reference's loop and for the necessary work (the device's form).  The
figures for the benchmark workload are frozen in
profiles/narrow_flops_per_stencil.txt, which bench.py reads.

    python oracle/count_flops.py            # C0 fold and the wavy-cloth strip
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from mclccd_b200 import scenes  # noqa: E402
from oracle.ref import Flops, Port  # noqa: E402


def count(V0, V1, F, eta):
    """Per-kind flop tallies over the oracle's candidate stencils of a scene
    and its hit rate; both counted forms must give port_accd's results."""
    p = Port().run(V0, V1, F, eta)
    kinds, (h, t), (hf, tf) = Flops().accd(V0, V1, p["cand_sten"], p["cand_is_vf"], eta)
    ph, pt = Port().accd(V0, V1, p["cand_sten"], p["cand_is_vf"], eta)
    assert np.array_equal(h, ph) and np.array_equal(t[ph == 1], pt[ph == 1])
    assert np.array_equal(hf, ph) and np.array_equal(tf[ph == 1], pt[ph == 1])
    return kinds, float(ph.mean())


def main():
    cases = [("folded cloth 64 x 64 (7,938 tris), thickness 1e-3", scenes.folded_cloth(64)),
             ("wavy cloth 1025 x 1025, strip of the first 257 rows (524,288 tris), thickness 1e-4",
              scenes.wavy_cloth(1025, seed=0, rows=257))]
    for name, (V0, V1, F, eta) in cases:
        kinds, rate = count(V0, V1, F, eta)
        print(f"# {name}: hit rate {rate:.3f}")
        for k in ("vf", "ee"):
            v = kinds[k]
            n = v["stencils"]
            print(f"#   {k}: {n} stencils, reference loop {v['reference_flops'] / n:.1f} flops/stencil "
                  f"({v['reference_distances'] / n:.2f} distances), necessary {v['necessary_flops'] / n:.1f}")


if __name__ == "__main__":
    main()
