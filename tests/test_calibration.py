"""Orientation binning of the calibration harness (CPU)."""
import numpy as np

from cpfem_code_b200 import calibration, generator


def test_bunge_matrix_matches_ctmatrx_layout():
    """bunge_matrix is the rotation the generator's compliance uses: S of a
    rotated crystal equals a^T-rotated S of the unrotated one."""
    rng = np.random.default_rng(0)
    eul = rng.random((5, 3)) * np.array([6.28, 3.14, 6.28])
    a = calibration.bunge_matrix(eul)
    for k in range(5):
        assert np.allclose(a[k] @ a[k].T, np.eye(3), atol=1e-14)
        assert abs(np.linalg.det(a[k]) - 1.0) < 1e-13
    e9 = generator.fcc_aluminium()["e"]
    S = generator.rotated_compliance(e9, eul)
    S0 = generator.rotated_compliance(e9, np.zeros((1, 3)))[0]
    # uniaxial compliance along the sample x axis = crystal direction a[:, 0]
    for k in range(5):
        d = a[k][:, 0]                       # sample x in the crystal frame
        s11 = S0[0, 0] * (d ** 4).sum() + (2 * S0[0, 1] + S0[3, 3]) * (
            d[0] ** 2 * d[1] ** 2 + d[1] ** 2 * d[2] ** 2 + d[2] ** 2 * d[0] ** 2)
        assert abs(S[k, 0, 0] - s11) < 1e-12 * abs(s11)


def test_cubic_families():
    assert len(calibration.cubic_family((1, 0, 0))) == 3
    assert len(calibration.cubic_family((1, 1, 0))) == 6
    assert len(calibration.cubic_family((1, 1, 1))) == 4
    assert len(calibration.cubic_family((3, 1, 1))) == 12


def test_bin_weights_select_aligned_grains():
    # the identity orientation has {100} normals along x, y, z; a 45-degree
    # rotation about z puts {110} along x
    eul = np.array([[0.0, 0.0, 0.0], [np.pi / 4, 0.0, 0.0], [0.3, 1.1, 0.7]])
    w100 = calibration.bin_weights(eul, calibration.cubic_family((1, 0, 0)), (1, 0, 0), 5.0)
    w110 = calibration.bin_weights(eul, calibration.cubic_family((1, 1, 0)), (1, 0, 0), 5.0)
    assert w100[0] == 1.0 and w100[1] == 0.0 and w100[2] == 0.0
    assert w110[1] == 1.0 and w110[0] == 0.0
    wide = calibration.bin_weights(eul, calibration.cubic_family((1, 0, 0)), (1, 0, 0), 50.0)
    assert abs(wide.sum() - 1.0) < 1e-15 and (wide > 0).sum() >= 2
