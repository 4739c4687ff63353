"""Structure factor on the GPU against the FP64 oracle and spsim's own outputs.

Tolerances (relative |F|^2 error against FP64, floored at 1e-3 of the mean
intensity, and L2 over the pattern; every path stores F and I as float32, so
one float ulp, ~6e-8, is the floor):
  fp64      2e-7  / 1e-7
  f32       1e-5  / 1e-6     FP64 or compensated FP32 phase, FMA-pipe sin/cos
  f32_fast  2e-4  / 1e-5     FP64 or compensated FP32 phase, MUFU sin/cos (the
                             neighbour-quad form: for half of each quad's
                             pixels, the others on the polynomials)
and against the reference's float results, its own error band (2e-5 / 2e-6).
"""
import numpy as np
import pytest
import torch

from conftest import golden, intensity_errors
from oracle import oracle as O
from spsim_b200 import core, synth

pytestmark = pytest.mark.gpu

TOL = {"fp64": (2e-7, 1e-7), "f32": (1e-5, 1e-6), "f32_fast": (2e-4, 1e-5)}
PRECS = ["fp64", "f32", "f32_fast"]


def _run(Z, pos, hkl, precision, **kw):
    B = kw.pop("B", 0.0)
    mol = core.Molecule(Z, pos, **kw)
    qs = core.QSet.from_list(hkl)
    F, I = core.forward(mol, qs, B=B, precision=precision)
    torch.cuda.synchronize()
    core.synchronize()
    return F.cpu().numpy().astype(np.complex128), I.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("precision", PRECS)
def test_small_molecule_against_fp64_and_reference(cuda, precision):
    g = golden("sf_small.npz")
    F64, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64))
    F, I = _run(g["Z"], g["pos"], g["hkl"], precision)
    e_max, e_l2 = intensity_errors(I, I64)
    print(precision, "vs FP64: floored max %.3g  L2 %.3g" % (e_max, e_l2))
    assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1]
    assert np.abs(F - F64).max() < 10 * TOL[precision][0] * np.abs(F64).max()
    r_max, r_l2 = intensity_errors(g["I"], I)  # the reference, measured against ours
    assert r_max < 2e-5 + TOL[precision][0] and r_l2 < 2e-6 + TOL[precision][1]


@pytest.mark.parametrize("precision", PRECS)
@pytest.mark.parametrize("variant,kw", [("_B20", {"B": 20.0}), ("_delta", {"delta_atoms": True})])
def test_b_factor_and_delta_atoms(cuda, precision, variant, kw):
    g = golden("sf_small.npz")
    F64, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64), **kw)
    F, I = _run(g["Z"], g["pos"], g["hkl"], precision, **kw)
    e_max, e_l2 = intensity_errors(I, I64)
    assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], (e_max, e_l2)
    r_max, _ = intensity_errors(g["I" + variant], I)
    assert r_max < 2e-5 + TOL[precision][0]


@pytest.mark.parametrize("precision", ["fp64", "f32"])
def test_gaussian_beam_illumination(cuda, precision):
    g = golden("sf_small.npz")
    beam = tuple(float(b) for b in g["beam"])
    F64, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64), beam=beam)
    F, I = _run(g["Z"], g["pos"], g["hkl"], precision, beam=beam)
    e_max, e_l2 = intensity_errors(I, I64)
    assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], (e_max, e_l2)


@pytest.mark.parametrize("precision", PRECS)
def test_plain_1k_workload_rows(cuda, precision):
    g = golden("sf_plain1k.npz")
    F64, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64))
    F, I = _run(g["Z"], g["pos"], g["hkl"], precision)
    e_max, e_l2 = intensity_errors(I, I64)
    print(precision, "plain_1k vs FP64: floored max %.3g  L2 %.3g" % (e_max, e_l2))
    assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1]
    r_max, r_l2 = intensity_errors(g["I"], I)
    assert r_max < 2e-5 + TOL[precision][0] and r_l2 < 2e-6 + TOL[precision][1]


@pytest.mark.parametrize("precision", ["f32", "f32_fast"])
def test_precision_stress_50k_subset(cuda, precision):
    # the 50,000-atom / 1024^2 workload on every 64th detector row: phases up to ~39 cycles
    w = synth.WORKLOADS["precision_50k"]
    Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
    d = w["det"]
    q64 = O.hkl_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    rows = np.arange(0, d["ny"], 64)
    sel = (rows[:, None] * d["nx"] + np.arange(d["nx"])[None, :]).reshape(-1)
    hkl = q64[sel].astype(np.float32)
    F64, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    F, I = _run(Z, pos, hkl, precision)
    e_max, e_l2 = intensity_errors(I, I64)
    print(precision, "precision_50k rows vs FP64: floored max %.3g  L2 %.3g" % (e_max, e_l2))
    assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1]


@pytest.mark.parametrize("precision", PRECS)
def test_edge_shapes(cuda, precision):
    rng = np.random.Generator(np.random.PCG64(9))
    for natoms, npix in [(1, 1), (7, 3), (9, 517), (130, 1), (257, 1031)]:
        Z = rng.choice([1, 6, 7, 8, 16, 26, 79], natoms).astype(np.int32)
        pos = (rng.normal(size=(natoms, 3)) * 1e-9).astype(np.float32)
        hkl = (rng.normal(size=(npix, 3)) * 3e8).astype(np.float32)
        F64, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
        F, I = _run(Z, pos, hkl, precision)
        assert np.abs(F - F64).max() <= 1e-5 * max(1.0, np.abs(F64).max()), (natoms, npix)


def test_empty_and_skipped_atoms(cuda):
    hkl = np.random.default_rng(1).normal(size=(100, 3)).astype(np.float32) * 1e8
    for Z in (np.zeros(0, np.int32), np.zeros(5, np.int32)):
        pos = np.zeros((len(Z), 3), np.float32)
        F, I = _run(Z, pos, hkl, "f32")
        assert np.all(F == 0) and np.all(I == 0)


def test_off_centre_molecule_phase(cuda):
    # a molecule 200 nm from the origin: F carries the exp(-2 pi i q.c) phase
    g = golden("sf_small.npz")
    pos = g["pos"].astype(np.float64) + np.array([2e-7, -1.5e-7, 0.7e-7])
    F64, I64 = O.structure_factor(g["Z"], pos, g["hkl"].astype(np.float64))
    F, I = _run(g["Z"], pos.astype(np.float32), g["hkl"], "f32")
    F64b, _ = O.structure_factor(g["Z"], pos.astype(np.float32).astype(np.float64), g["hkl"].astype(np.float64))
    e_max, e_l2 = intensity_errors(I, np.abs(F64b) ** 2)
    assert e_max < 1e-5 and e_l2 < 1e-6
    assert np.abs(F - F64b).max() < 1e-4 * np.abs(F64b).max()


@pytest.mark.parametrize("precision", ["f32", "fp64"])
def test_rotation_and_detector_qset(cuda, precision):
    w = synth.WORKLOADS["orientations_20k"]
    Z, pos = synth.random_molecule(2000, 3e-9, 77)
    d = w["det"]
    R = synth.haar_rotations(3, 5)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(64, 64, d["width"] / 4, d["height"] / 4, d["distance"], d["wavelength"])
    q0 = O.hkl_detector(64, 64, d["width"] / 4, d["height"] / 4, d["distance"], d["wavelength"])
    for r in R:
        F, I = core.forward(mol, qs, rot=r, precision=precision)
        F64, I64 = O.structure_factor(Z, pos.astype(np.float64), q0 @ r.T)
        e_max, e_l2 = intensity_errors(I.cpu().numpy(), I64)
        assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], (e_max, e_l2)


def test_batch_equals_single_patterns(cuda):
    rng = np.random.Generator(np.random.PCG64(3))
    mols, qsets, ref = [], [], []
    for i, (n, nx) in enumerate([(300, 24), (1500, 40), (64, 16), (4000, 8)]):
        Z, pos = synth.random_molecule(n, (n / 50e27 * 3 / 4 / np.pi) ** (1 / 3), 40 + i)
        m = core.Molecule(Z, pos)
        q = core.QSet.from_detector(nx, nx, nx * 150e-6, nx * 150e-6, 0.1, 0.2e-9)
        mols.append(m)
        qsets.append(q)
        ref.append(core.forward(m, q, precision="f32")[1].clone())
    R = np.stack([np.eye(3)] * 4)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):  # a non-default stream: captured once, then graph-replayed
        F, I = core.forward_batch(mols, qsets, rots=R, precision="f32")
        F2, I2 = core.forward_batch(mols, qsets, rots=R, precision="f32")
    s.synchronize()
    core.synchronize(s)
    for a, b, c in zip(I, I2, ref):
        torch.testing.assert_close(a, c, rtol=1e-6, atol=1e-6 * float(c.abs().max()))
        torch.testing.assert_close(b, c, rtol=1e-6, atol=1e-6 * float(c.abs().max()))


def test_range_error_is_reported(cuda):
    # a 2 um object at 3e9 1/m (6000 cycles) is outside the compensated kernels'
    # phase domain; the FP64-phase form (the default) has no such limit
    Z = np.array([6, 6], np.int32)
    pos = np.array([[-1e-6, 0, 0], [1e-6, 0, 0]], np.float32)
    mol = core.Molecule(Z, pos)
    hkl = np.array([[3e9, 0, 0], [2.9e9, 1e8, 3e7]], np.float32)
    qs = core.QSet.from_list(hkl)
    from spsim_b200._native import SpsimError, SPSIM_ERR_RANGE

    F64, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    try:
        for form in (0, 1):
            core.set_variant(128, 4, form)
            with pytest.raises(SpsimError) as e:
                core.forward(mol, qs, precision="f32")
            assert e.value.status == SPSIM_ERR_RANGE
        core.set_variant(128, 4, 2)
        F, I = core.forward(mol, qs, precision="f32")
        assert np.abs(I.cpu().numpy() - I64).max() < 1e-5 * I64.max()
    finally:
        core.set_variant(-1)
    F, I = core.forward(mol, qs, precision="fp64")
    assert np.abs(I.cpu().numpy() - I64).max() < 2e-7 * I64.max()


@pytest.mark.parametrize("precision", ["f32", "f32_fast"])
def test_wide_phase_range_uses_fp64_rounding(cuda, precision):
    # |q|max |r - c|max of ~6e5 cycles is above the fixed-point phase word's
    # 2^17-cycle range: the FP64-phase forms reduce by FP64 rounding instead
    rng = np.random.Generator(np.random.PCG64(5))
    Z = rng.choice([6, 7, 8, 16], 64).astype(np.int32)
    pos = rng.uniform(-3e-5, 3e-5, (64, 3)).astype(np.float32)
    # pixel pairs 2m, 2m+1 a few 100 1/m apart, so that the neighbour-pair form is admitted too
    qa = rng.normal(size=(1024, 3)) * 3e9
    hkl = np.stack([qa, qa + rng.normal(size=(1024, 3)) * 3e2], axis=1).reshape(-1, 3).astype(np.float32)
    qr = np.linalg.norm(hkl.astype(np.float64), axis=1).max() * np.linalg.norm(pos - pos.mean(0), axis=1).max()
    assert qr > 2.0 ** 17
    _, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    for form in (2, 3):
        try:
            core.set_variant(128, 4, form)
            _, I = _run(Z, pos, hkl, precision)
            assert core.last_variant()[2] == form and not core.last_phase_word()
        finally:
            core.set_variant(-1)
        e_max, e_l2 = intensity_errors(I, I64)
        assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], (form, e_max, e_l2)


VARIANTS = [(128, 2, 0), (256, 4, 0), (128, 4, 1), (128, 6, 1), (128, 2, 2), (128, 4, 2), (256, 4, 2), (128, 8, 2),
            (128, 4, 3), (128, 8, 3), (128, 12, 3), (256, 4, 3), (128, 8, 4), (128, 16, 4), (256, 8, 4)]


@pytest.mark.parametrize("precision", ["f32", "f32_fast"])
@pytest.mark.parametrize("variant", VARIANTS, ids=["%dx%d_form%d" % v for v in VARIANTS])
def test_every_kernel_form_meets_tolerance(cuda, precision, variant):
    # each compiled variant, forced, on the plain 1k workload (whole detector
    # rows: pairs and quads are admitted) and with per-atom B factors
    g = golden("sf_plain1k.npz")
    F64, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64))
    rng = np.random.Generator(np.random.PCG64(17))
    bfac = rng.uniform(0, 40, len(g["Z"])).astype(np.float32)
    F64b, I64b = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64), bfac=bfac)
    try:
        core.set_variant(*variant)
        F, I = _run(g["Z"], g["pos"], g["hkl"], precision)
        assert core.last_variant() == variant
        Fb, Ib = _run(g["Z"], g["pos"], g["hkl"], precision, bfac=bfac)
        assert core.last_variant() == variant
    finally:
        core.set_variant(-1)
    for got, want in ((I, I64), (Ib, I64b)):
        e_max, e_l2 = intensity_errors(got, want)
        assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], (variant, e_max, e_l2)


def test_neighbour_form_admission(cuda):
    # a detector of width divisible by 4 is admitted to the neighbour-quad
    # form, one of even width (6: quads straddle rows) to the neighbour-pair
    # form; a random HKL list (no neighbour structure) falls back to the
    # FP64-phase form; all stay within tolerance
    Z, pos = synth.random_molecule(2000, 3e-9, 31)
    d = dict(nx=64, ny=40, width=64 * 150e-6, height=40 * 150e-6, distance=0.1, wavelength=0.2e-9)
    q_det = O.hkl_detector(**d).astype(np.float32)
    d6 = dict(nx=6, ny=400, width=6 * 150e-6, height=400 * 150e-6, distance=0.1, wavelength=0.2e-9)
    q_det6 = O.hkl_detector(**d6).astype(np.float32)
    q_rand = np.random.Generator(np.random.PCG64(31)).normal(size=(2560, 3)).astype(np.float32) * 1e9
    for q, kernel in ((q_det, "sf_dquad_kernel"), (q_det6, "sf_dpair_kernel"), (q_rand, "sf_dphase_kernel")):
        F, I = _run(Z, pos, q, "f32")
        assert core.kernel_name() == kernel and core.last_phase_word()
        _, I64 = O.structure_factor(Z, pos.astype(np.float64), q.astype(np.float64))
        e_max, e_l2 = intensity_errors(I, I64)
        assert e_max < TOL["f32"][0] and e_l2 < TOL["f32"][1], (kernel, e_max, e_l2)


@pytest.mark.parametrize("step,narrow", [(0.065, True), (0.11, False)])
def test_neighbour_pair_step_selects_second_pixel_polynomial(cuda, step, narrow):
    # pairs whose step |q_b - q_a| times the molecule's bound (its bounding-box
    # radius plus the refinement margin) stays within 0.07 cycle evaluate the
    # second pixel with the shorter NARROW polynomial; steps up to 1/8 cycle
    # keep the WIDE one; both stay within tolerance, on the steepest step the
    # admission allows, with and without per-atom B factors
    Z, pos = synth.random_molecule(3000, 3e-9, 41)
    p64 = pos.astype(np.float64)
    c = 0.5 * (p64.min(0) + p64.max(0))
    rmax = np.linalg.norm(p64 - c, axis=1).max()
    rbound = rmax + max(0.05 * rmax, 5e-10)
    rng = np.random.Generator(np.random.PCG64(42))
    qa = rng.normal(size=(4096, 3)) * 1.5e9
    u = rng.normal(size=(4096, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    hkl = np.stack([qa, qa + u * (step / rbound)], axis=1).reshape(-1, 3).astype(np.float32)
    bfac = rng.uniform(0, 40, len(Z)).astype(np.float32)
    for kw in ({}, {"bfac": bfac}):
        _, I64 = O.structure_factor(Z, p64, hkl.astype(np.float64), **kw)
        try:
            core.set_variant(128, 8, 3)
            _, I = _run(Z, pos, hkl, "f32", **kw)
            assert core.kernel_name() == "sf_dpair_kernel" and core.last_phase_word()
            assert core.last_pair_narrow() == narrow
        finally:
            core.set_variant(-1)
        e_max, e_l2 = intensity_errors(I, I64)
        assert e_max < TOL["f32"][0] and e_l2 < TOL["f32"][1], (step, kw.keys(), e_max, e_l2)
        _, I = _run(Z, pos, hkl, "f32_fast", **kw)
        assert not core.last_pair_narrow()  # the MUFU forms have no polynomial


def _quads(rng, n, s1, s2, scale=1.5e9):
    """A q list of n quads 4m..4m+3 around random anchors q_a = q[4m+1]: the
    one-pixel neighbours at distance s1 (in 1/m), the two-pixel one at s2."""
    qa = rng.normal(size=(n, 3)) * scale
    u = rng.normal(size=(n, 3, 3))
    u /= np.linalg.norm(u, axis=2, keepdims=True)
    return np.stack([qa + u[:, 0] * s1, qa, qa + u[:, 1] * s1, qa + u[:, 2] * s2], axis=1).reshape(-1, 3)


def _bound(pos):
    p64 = pos.astype(np.float64)
    c = 0.5 * (p64.min(0) + p64.max(0))
    rmax = np.linalg.norm(p64 - c, axis=1).max()
    return rmax + max(0.05 * rmax, 5e-10)


@pytest.mark.parametrize("step1,step2,narrow", [(0.065, 0.155, True), (0.12, 0.155, False)])
def test_neighbour_quad_steps_select_polynomials(cuda, step1, step2, narrow):
    # quads whose one-pixel steps (times the molecule's bound) stay within
    # 0.07 cycle take the NARROW polynomial for them, up to 1/8 the WIDER one;
    # the two-pixel step always takes WIDER (up to 0.16); all within tolerance
    # on the steepest steps the admission allows, with and without B factors
    Z, pos = synth.random_molecule(3000, 3e-9, 43)
    rb = _bound(pos)
    rng = np.random.Generator(np.random.PCG64(44))
    hkl = _quads(rng, 2048, step1 / rb, step2 / rb).astype(np.float32)
    bfac = rng.uniform(0, 40, len(Z)).astype(np.float32)
    for kw in ({}, {"bfac": bfac}):
        _, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64), **kw)
        _, I = _run(Z, pos, hkl, "f32", **kw)
        assert core.kernel_name() == "sf_dquad_kernel" and core.last_phase_word()
        assert core.last_pair_narrow() == narrow
        e_max, e_l2 = intensity_errors(I, I64)
        assert e_max < TOL["f32"][0] and e_l2 < TOL["f32"][1], (step1, kw.keys(), e_max, e_l2)


def test_fast_mode_takes_the_split_pipe_quads(cuda):
    # f32_fast on a detector q set runs the quad form with pixels 4m+2, 4m+3 on
    # MUFU (all on polynomials in f32), within its tolerance, with and without
    # per-atom B factors (one MUFU pixel per quad there)
    Z, pos = synth.random_molecule(3000, 3e-9, 48)
    d = dict(nx=64, ny=48, width=64 * 150e-6, height=48 * 150e-6, distance=0.1, wavelength=0.2e-9)
    hkl = O.hkl_detector(**d).astype(np.float32)
    bfac = np.random.Generator(np.random.PCG64(49)).uniform(0, 40, len(Z)).astype(np.float32)
    for kw in ({}, {"bfac": bfac}):
        _, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64), **kw)
        for precision in ("f32", "f32_fast"):
            _, I = _run(Z, pos, hkl, precision, **kw)
            assert core.kernel_name() == "sf_dquad_kernel" and core.last_pair_narrow()
            e_max, e_l2 = intensity_errors(I, I64)
            assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], (precision, kw.keys(), e_max, e_l2)


def test_neighbour_quad_admission_limits(cuda):
    # a two-pixel step beyond 0.16 cycle, or a one-pixel step beyond 1/8,
    # sends the q set to the pair form (or form 2) instead
    Z, pos = synth.random_molecule(1000, 2e-9, 45)
    rb = _bound(pos)
    rng = np.random.Generator(np.random.PCG64(46))
    for s1, s2 in ((0.05, 0.17), (0.13, 0.1)):
        hkl = _quads(rng, 512, s1 / rb, s2 / rb).astype(np.float32)
        _, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
        _, I = _run(Z, pos, hkl, "f32")
        assert core.kernel_name() != "sf_dquad_kernel", (s1, s2)
        e_max, e_l2 = intensity_errors(I, I64)
        assert e_max < TOL["f32"][0] and e_l2 < TOL["f32"][1]


@pytest.mark.parametrize("npix", [1, 2, 3, 5, 6, 7, 1021, 1022, 1023, 1029])
def test_neighbour_quads_with_a_partial_last_quad(cuda, npix):
    # q sets whose length is not a multiple of 4 (and tiles that end inside a
    # quad): the last quad anchors on its first pixel when that is its only one
    Z, pos = synth.random_molecule(700, 2e-9, 47)
    d = dict(nx=64, ny=20, width=64 * 150e-6, height=20 * 150e-6, distance=0.1, wavelength=0.2e-9)
    hkl = O.hkl_detector(**d)[:npix].astype(np.float32)
    _, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    for variant in ((128, 8, 4), (128, 16, 4), (256, 8, 4)):
        try:
            core.set_variant(*variant)
            _, I = _run(Z, pos, hkl, "f32")
            assert core.last_variant() == variant
        finally:
            core.set_variant(-1)
        e_max, e_l2 = intensity_errors(I, I64)
        assert e_max < TOL["f32"][0] and e_l2 < TOL["f32"][1], (npix, variant, e_max, e_l2)


CANDIDATES = {(128, 2, 0), (128, 4, 0), (256, 4, 0), (128, 2, 1), (128, 4, 1), (256, 4, 1), (128, 6, 1), (128, 2, 2),
              (128, 4, 2), (256, 4, 2), (128, 6, 2), (128, 8, 2), (128, 4, 3), (128, 8, 3), (128, 12, 3), (256, 4, 3),
              (128, 8, 4), (128, 16, 4), (256, 8, 4)}


def test_autotune_single_and_batch(cuda):
    # the autotuners time every compiled variant, keep the fastest for the
    # workload's size class, and the forwards that follow use it and stay
    # within tolerance; clearing the tuning restores the untuned defaults
    Z, pos = synth.random_molecule(1500, 2.5e-9, 61)
    d = dict(nx=48, ny=40, width=48 * 150e-6, height=40 * 150e-6, distance=0.1, wavelength=0.2e-9)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(**d)
    q = O.hkl_detector(**d)
    R = synth.haar_rotations(3, 62)
    try:
        best = core.autotune(mol, qs, precision="f32")
        assert best in CANDIDATES
        _, I = core.forward(mol, qs, precision="f32")
        assert core.last_variant()[:2] == best[:2]
        _, I64 = O.structure_factor(Z, pos.astype(np.float64), q)
        e_max, e_l2 = intensity_errors(I.cpu().numpy(), I64)
        assert e_max < TOL["f32"][0] and e_l2 < TOL["f32"][1]
        best_b = core.autotune_batch([mol] * 3, [qs] * 3, rots=R, precision="f32")
        assert best_b in CANDIDATES
        _, Ib = core.forward_batch([mol] * 3, [qs] * 3, rots=R, precision="f32")
        assert core.last_variant()[:2] == best_b[:2]
        for r, Ir in zip(R, Ib):
            _, I64r = O.structure_factor(Z, pos.astype(np.float64), q @ r.T)
            e_max, e_l2 = intensity_errors(Ir.cpu().numpy(), I64r)
            assert e_max < TOL["f32"][0] and e_l2 < TOL["f32"][1]
    finally:
        core.clear_tuning()
    core.forward(mol, qs, precision="f32")
    assert core.last_variant() == (128, 8, 4)  # the untuned default again


@pytest.mark.parametrize("form", [2, 3])
def test_b_factors_with_negative_and_zero_occupancies(cuda, form):
    # per-atom B factors fold the atom weight into the exponent, exp2(b s^2 +
    # log2|w|), and carry the weight's sign as an extra half cycle of phase:
    # negative and zero occupancies (refinement can produce both) must come out
    # as with the plain product
    g = golden("sf_plain1k.npz")
    rng = np.random.Generator(np.random.PCG64(71))
    n = len(g["Z"])
    occ = rng.uniform(-0.6, 1.0, n).astype(np.float32)
    occ[::17] = 0.0
    bfac = rng.uniform(0, 40, n).astype(np.float32)
    _, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64), occ=occ, bfac=bfac)
    try:
        core.set_variant(128, 4, form)
        _, I = _run(g["Z"], g["pos"], g["hkl"], "f32", occ=occ, bfac=bfac)
        assert core.last_variant()[2] == form and core.last_phase_word()
    finally:
        core.set_variant(-1)
    e_max, e_l2 = intensity_errors(I, I64)
    assert e_max < TOL["f32"][0] and e_l2 < TOL["f32"][1], (e_max, e_l2)


def test_atoms_moved_outside_bounds_are_reported(cuda):
    # refinement moves past the creation-time radius (and its margin) are
    # reported as SPSIM_ERR_RANGE by the next forward's synchronisation, for
    # cached (graph) and FP64 plans alike; moving back clears it
    from spsim_b200._native import SpsimError, SPSIM_ERR_RANGE

    Z, pos = synth.random_molecule(300, 1e-9, 16)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_list((np.random.default_rng(4).normal(size=(700, 3)) * 1e9).astype(np.float32))
    moved = pos.astype(np.float64).copy()
    moved[5] += 3e-8
    for precision in ("f32", "fp64"):
        mol.update_device(torch.from_numpy(moved).cuda())
        core.forward(mol, qs, precision=precision)
        with pytest.raises(SpsimError) as e:
            core.synchronize()
        assert e.value.status == SPSIM_ERR_RANGE
        mol.update_device(torch.from_numpy(pos.astype(np.float64)).cuda())
        _, I = core.forward(mol, qs, precision=precision)
        core.synchronize()
        _, I64 = O.structure_factor(Z, pos.astype(np.float64), qs.q().astype(np.float64))
        e_max, _ = intensity_errors(I.cpu().numpy(), I64)
        assert e_max < 1e-5
