"""The FP64 oracle pinned against spsim's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference sources) and against published
known answers.  CPU only."""
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden, intensity_errors
from oracle import oracle as O


def _product_table():
    text = open(os.path.join(ROOT, "spsim_b200", "csrc", "atomsf_data.h")).read()
    rows = re.findall(r"\{([-0-9.e+f, ]+)\}", text)
    return np.array([[float(v.strip().rstrip("f")) for v in r.split(",")] for r in rows], np.float32)


def test_form_factor_table_is_the_reference_table():
    ref = np.load(os.path.join(GOLDEN, "atomsf_reference.npy"))
    assert ref.shape == (100, 9)
    np.testing.assert_array_equal(_product_table(), ref)


def test_scatt_factor_at_zero_q_is_sum_of_coefficients():
    ref = np.load(os.path.join(GOLDEN, "atomsf_reference.npy"))
    for z in (1, 6, 7, 8, 16, 26, 79):
        assert O.scatt_factor(0.0, z) == pytest.approx(float(np.sum(ref[z, :4].astype(np.float64)) + ref[z, 8]),
                                                       rel=1e-12)


def test_scatt_factor_b_factor_factorises():
    # f(q, B) = exp(-B s^2) f(q, 0), s = |q| 1e-10 / 2 (src/diffraction.c:183-193)
    q = 3.1e9
    s2 = (q * 1e-10) ** 2 / 4
    assert O.scatt_factor(q, 8, 25.0) == pytest.approx(np.exp(-25.0 * s2) * O.scatt_factor(q, 8, 0.0), rel=1e-12)


@pytest.mark.parametrize("spherical", [False, True])
def test_hkl_list_matches_reference_bit_for_bit(spherical):
    g = golden("sf_small.npz")
    nx, ny, w, h, d, lam = g["det"]
    q = O.hkl_detector(int(nx), int(ny), w, h, d, lam, spherical=spherical)
    ref = g["hkl_spherical"] if spherical else g["hkl"]
    np.testing.assert_array_equal(q.astype(np.float32), ref)


def _fp64_of(g, **kw):
    return O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64), **kw)


# The reference computes the phase and the sum in float (src/diffraction.c:836-839),
# so it agrees with the FP64 restatement only to float accuracy: these bounds are
# the reference's own error, measured, with a margin.
@pytest.mark.parametrize("variant,kw,tol_max,tol_l2", [
    ("", {}, 2e-5, 2e-6),
    ("_B20", {"B": 20.0}, 2e-5, 2e-6),
    ("_delta", {"delta_atoms": True}, 2e-5, 2e-6),
])
def test_structure_factor_oracle_matches_reference(variant, kw, tol_max, tol_l2):
    g = golden("sf_small.npz")
    F64, I64 = _fp64_of(g, **kw)
    e_max, e_l2 = intensity_errors(g["I" + variant], I64)
    assert e_max < tol_max and e_l2 < tol_l2, (e_max, e_l2)
    np.testing.assert_allclose(g["F" + variant], F64, atol=2e-6 * np.abs(F64).max())


def test_structure_factor_oracle_matches_reference_gaussian_beam():
    g = golden("sf_small.npz")
    F64, I64 = _fp64_of(g, beam=tuple(g["beam"]))
    e_max, e_l2 = intensity_errors(g["I_beam"], I64)
    assert e_max < 2e-5 and e_l2 < 2e-6, (e_max, e_l2)


def test_structure_factor_oracle_matches_reference_sse_path():
    # the SSE path does not skip Z = 0 atoms (src/diffraction.c:903-957): one
    # atom of this molecule has Z = 0 and contributes f = -1 there
    g = golden("sf_small.npz")
    Z = g["Z"].copy()
    assert (Z == 0).sum() == 1
    F64, I64 = _fp64_of(g)
    zero = np.where(Z == 0)[0][0]
    q = g["hkl"].astype(np.float64)
    ph = q @ g["pos"][zero].astype(np.float64)
    F_sse = F64 - np.exp(-2j * np.pi * ph)
    e_max, e_l2 = intensity_errors(g["I_vector"], np.abs(F_sse) ** 2)
    assert e_max < 2e-5 and e_l2 < 2e-6, (e_max, e_l2)


def test_plain_1k_workload_subset_matches_reference():
    g = golden("sf_plain1k.npz")
    F64, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64))
    e_max, e_l2 = intensity_errors(g["I"], I64)
    assert e_max < 2e-5 and e_l2 < 2e-6, (e_max, e_l2)


def _chain_params(g):
    p = g["params"]
    keys = ["nx", "ny", "width", "height", "distance", "pw", "ph", "cx", "cy", "qe", "ehole", "dark", "fullwell",
            "maxv", "bx", "by", "lam", "I0", "t"]
    return dict(zip(keys, p))


def test_geometry_factors_match_reference():
    g = golden("chain.npz")
    c = _chain_params(g)
    nx, ny = int(c["nx"]), int(c["ny"])
    for pol in range(4):
        T = O.thomson(nx, ny, c["width"], c["height"], c["distance"], pol, c["cx"], c["cy"])
        np.testing.assert_array_equal(T.astype(np.float32), g["thomson_%d" % pol])
    for sph in (0, 1):
        S = O.solid_angle(nx, ny, c["width"], c["height"], c["distance"], c["pw"], c["ph"], bool(sph), c["cx"], c["cy"])
        np.testing.assert_allclose(S.astype(np.float32), g["solid_angle_%d" % sph], rtol=2e-7)


def test_photon_electron_and_binned_outputs_match_reference():
    g = golden("chain.npz")
    c = _chain_params(g)
    nx, ny = int(c["nx"]), int(c["ny"])
    photons = (g["thomson_3"] * g["solid_angle_0"] * g["ints"] * np.float32(c["I0"])).astype(np.float32)
    np.testing.assert_allclose(photons, g["photons"], rtol=1e-6)
    hc = 1.98644521e-25
    epp = np.float32((hc / np.float64(np.float32(c["lam"]))) / np.float64(np.float32(c["ehole"])))
    np.testing.assert_array_equal((g["counts"] * epp).astype(np.float32), g["electrons"])
    nl = O.noiseless_output(g["photons"], nx, ny, int(c["bx"]), int(c["by"]), np.float32(c["qe"]),
                            np.float32(c["lam"]), np.float32(c["ehole"]), c["fullwell"], c["maxv"])
    np.testing.assert_allclose(nl, g["noiseless_output"], rtol=1e-6)
    ro = O.real_output(g["electrons"], None, nx, ny, int(c["bx"]), int(c["by"]), np.float32(c["dark"]),
                       np.float32(c["t"]), c["fullwell"], c["maxv"])
    np.testing.assert_allclose(ro, g["real_output"], rtol=1e-6)


# Random123 known-answer vectors for Philox4x32-10 (Salmon et al., SC'11)
@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0, 0, 0), 0, (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, 0xffffffffffffffff, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0x299f31d0 << 32) | 0xa4093822,
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(ctr, key, expect):
    assert tuple(int(x) for x in O.philox(*ctr, key)) == expect


def test_oracle_poisson_moments():
    lam = np.repeat(np.array([0.3, 4.0, 25.0, 400.0, 5000.0], np.float32), 40000)
    k = O.poisson(lam, seed=12345).reshape(5, -1)
    for i, l in enumerate([0.3, 4.0, 25.0, 400.0, 5000.0]):
        m, v = k[i].mean(), k[i].var()
        se = np.sqrt(l / k.shape[1])
        assert abs(m - l) < 5 * se + 0.5 * (l >= 1000), (l, m)
        assert abs(v / l - 1) < 0.05, (l, v)
