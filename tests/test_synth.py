"""Synthetic workload generators."""
import numpy as np

from spsim_b200 import synth


def test_composition_counts_exact():
    c = synth.composition_counts(1000)
    assert c == {6: 620, 7: 170, 8: 200, 16: 10}
    assert sum(synth.composition_counts(12345).values()) == 12345


def test_random_molecule_ball_and_separation():
    from scipy.spatial import cKDTree

    Z, pos = synth.random_molecule(2000, 2.5e-9, 3)
    assert Z.shape == (2000,) and pos.shape == (2000, 3) and pos.dtype == np.float32
    assert np.linalg.norm(pos.astype(np.float64), axis=1).max() <= 2.5e-9 * (1 + 1e-6)
    d, _ = cKDTree(pos.astype(np.float64)).query(pos.astype(np.float64), k=2)
    assert d[:, 1].min() >= synth.MIN_SEPARATION * (1 - 1e-5)
    Z2, pos2 = synth.random_molecule(2000, 2.5e-9, 3)
    assert np.array_equal(Z, Z2) and np.array_equal(pos, pos2)


def test_haar_rotations_orthonormal_and_uniform():
    R = synth.haar_rotations(2000, 5)
    I = np.einsum("nij,nkj->nik", R, R)
    assert np.abs(I - np.eye(3)).max() < 1e-12
    assert np.allclose(np.linalg.det(R), 1)
    # the image of the z axis is uniform on the sphere: mean ~ 0, <z^2> ~ 1/3
    v = R[:, :, 2]
    assert np.abs(v.mean(0)).max() < 0.06
    assert abs((v[:, 2] ** 2).mean() - 1 / 3) < 0.03


def test_uneven_batch_shapes():
    mols = synth.uneven_batch()
    assert len(mols) == 64
    n = np.array([m["natoms"] for m in mols])
    assert n.min() >= 500 and n.max() <= 100000
    assert {m["det"]["nx"] for m in mols} <= {128, 256, 512, 1024}
