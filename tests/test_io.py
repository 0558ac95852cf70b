"""Fixture/result I/O in the reference's text formats and the timing statistics
of its notebook (no GPU)."""
import numpy as np

from conftest import golden
from cugmres_b200 import io


def test_complex_roundtrip_matches_fixture_values(tmp_path):
    """Lines in the reference's "re im" format (values of G_prep_32.txt) read back exactly."""
    g = golden("ref_G_prep_32.npz")
    key = [k for k in g.files if g[k].dtype.kind == "c"][0]
    vals = g[key].reshape(-1)[:50]
    p = tmp_path / "G_prep.txt"
    io.write_complex_txt(p, vals)
    back = io.read_complex_txt(p)
    assert np.max(np.abs(back - vals)) <= 1e-11 * np.max(np.abs(vals))
    # the reference's own line layout: two numbers separated by one space
    first = open(p).readline().split()
    assert len(first) == 2


def test_mask_roundtrip(tmp_path):
    m = golden("ref_cylinder_32.npz")
    mask = np.unpackbits(m["mask"])[: 32 * 32].astype(bool)  # stored bit-packed
    p = tmp_path / "cylinder_32.txt"
    io.write_mask_txt(p, mask)
    assert set(open(p).read().split()) <= {"0", "1"}
    assert np.array_equal(io.read_mask_txt(p, 32), mask.reshape(32, 32))


def test_grid_and_results(tmp_path):
    a = (np.arange(16) + 1j * np.arange(16)[::-1]).reshape(4, 4)
    p = tmp_path / "a.txt"
    io.write_complex_txt(p, a)
    assert np.array_equal(io.read_grid(p, 4), a)
    io.save_results(tmp_path / "r.npz", x=a, iterations=17, res_hist=np.array([1.0, 0.5]))
    r = io.load_results(tmp_path / "r.npz")
    assert np.array_equal(r["x"], a) and int(r["iterations"]) == 17


def test_refined_statistics():
    x = np.array([10.0, 10.2, 9.8, 10.1, 30.0])
    mean, std = io.refined_stats(x)
    assert abs(std - np.std(x)) < 1e-12
    assert abs(mean - np.mean([10.0, 10.2, 9.8, 10.1])) < 1e-12  # the outlier is dropped
    # no sample within one std of the mean: the plain mean
    y = np.array([0.0, 2.0])
    assert io.refined_stats(y)[0] == 1.0
    assert np.array_equal(io.step_durations([0, 5, 9, 0, 20]), [4, 11])
