"""Input forms other than row-major double (mclccd_update_ex /
mclccd_traverse_ex): column-major V and P (Eigen's default MatrixXd /
MatrixXi layouts) and float coordinates are passed as they are and
converted on the device.  The results equal those of row-major double
inputs holding the same values."""
import numpy as np
import pytest

from mclccd_b200 import BVHTree, ccd, scenes


def test_layout_detection_takes_arrays_as_they_are():
    V = np.asfortranarray(np.random.default_rng(0).random((50, 3)))
    F = np.asfortranarray(np.arange(30, dtype=np.int32).reshape(10, 3))
    assert ccd._colmajor(V, np.float64) and ccd._colmajor(F, np.int32)
    assert not ccd._colmajor(np.ascontiguousarray(V), np.float64)
    assert not ccd._colmajor(V.astype(np.float32, order="F"), np.float64)
    assert ccd._colmajor(V.astype(np.float32, order="F"), np.float32)
    ptr, kind, keep, rows = ccd._arg_colmajor(V)
    assert keep is V and ptr.value == V.ctypes.data and rows == 50 and kind == ccd.MEM_HOST


def run(V0, V1, F, eta, dim):
    t = BVHTree(dim)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    s, v, toi = t.hits()
    first = {(int(a),) + tuple(map(int, b)): float(c) for b, a, c in zip(s, v, toi)}
    t.update(V0, V1, F)   # refit-only step on the update's arrays
    t.traverse()
    s, v, toi = t.hits()
    again = {(int(a),) + tuple(map(int, b)): float(c) for b, a, c in zip(s, v, toi)}
    assert again == first
    return first, np.sort(t.discrete(), axis=0)


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["fold", "annulus"])
def test_column_major_and_float_inputs(scene):
    torch = pytest.importorskip("torch")
    V0, V1, F, eta = scenes.folded_cloth(36, seed=51) if scene == "fold" else scenes.annulus_2d(300, seed=52)
    dim = V0.shape[1]
    want, wd = run(V0, V1, F, eta, dim)
    assert len(want) > 0
    cases = {
        "numpy F-order V and P": (np.asfortranarray(V0), np.asfortranarray(V1), np.asfortranarray(F)),
        "numpy F-order V only": (np.asfortranarray(V0), np.asfortranarray(V1), F),
        "numpy F-order P only": (V0, V1, np.asfortranarray(F)),
        "CUDA column-major views": tuple(torch.from_numpy(np.ascontiguousarray(x.T)).cuda().T for x in (V0, V1, F)),
    }
    for name, (a0, a1, aF) in cases.items():
        got, gd = run(a0, a1, aF, eta, dim)
        assert got == want, name
        assert np.array_equal(gd, wd), name
    # float coordinates, column-major, against the row-major double run on
    # the same (widened) values
    f0, f1 = V0.astype(np.float32), V1.astype(np.float32)
    feta = float(np.float32(eta))
    want32, _ = run(f0.astype(np.float64), f1.astype(np.float64), F, feta, dim)
    got32, _ = run(np.asfortranarray(f0), np.asfortranarray(f1), np.asfortranarray(F), feta, dim)
    assert got32 == want32
