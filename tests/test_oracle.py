"""The CPU oracle against the reference's known answers and against itself.

These run without a GPU.  They pin the oracle (the checker of every GPU
parity test) to the reference: the shipped synthesis vector
data/synthesis_gpu.per (tests/golden/kat_synthesis.npz), finite differences
of its own synthesis, and the algebra of its solver.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O


def kat_cfg():
    g = H.kat()
    l0 = float(g["lambda0"])
    z = O.cuanten(*g["quantum"], 1.0)
    first, step, last = g["grid"]
    lam = O.grid_lambda(l0, first, step, last)
    off = O.grid_offsets_mA(first, step, last)
    psf = O.psf_from_table(g["psf_x_mA"], g["psf_y"], off, step)
    return g, O.make_cfg(lam, l0, z, psf=psf, mu=float(g["mu"])), off


def test_kat_grid_and_line():
    g, cfg, off = kat_cfg()
    assert cfg.nl == 30
    np.testing.assert_allclose(off, g["per_offsets_mA"], atol=1e-6)
    assert cfg.z.n_pi == 1 and cfg.z.n_sig == 1
    assert cfg.z.geff == pytest.approx(2.5)
    assert list(cfg.z.nub)[:1] == [-2.5] and list(cfg.z.nur)[:1] == [2.5]


@pytest.mark.parametrize("mode", ["faithful_f32", "fp64"])
def test_kat_synthesis(mode):
    """Reference known answer: synthesis of run/init.mod with the CRISP PSF.
    The file holds 7 significant digits; agreement is limited by that."""
    g, cfg, _ = kat_cfg()
    fn = O.synth_f if mode == "faithful_f32" else O.synth_d
    s = fn(cfg, g["model"])
    rel = H.normwise(s, g["per_iquv"])
    assert rel.max() < 2e-6, rel


def test_kat_psf_is_centred_and_normalised():
    g, cfg, _ = kat_cfg()
    psf = np.array(cfg.psf[:cfg.nl])
    assert psf.sum() == pytest.approx(1.0, abs=1e-12)
    assert psf.argmax() == cfg.nl // 2


@pytest.fixture
def mo_scale_exact():
    O.lib().orc_set_mo_scale(2.0)
    yield
    O.lib().orc_set_mo_scale(1.0)


@pytest.mark.parametrize("use_psf", [False, True])
def test_rf_finite_differences(use_psf, mo_scale_exact):
    """Analytic response functions against central differences of the FP64
    synthesis.  With the dispersion derivatives doubled (the reference halves
    them, see the next test) every RF matches to the accuracy of the Voigt
    approximation's derivative relations."""
    g, cfg, _ = kat_cfg()
    if not use_psf:
        cfg.use_psf = 0
    m = g["model"].copy()
    _, rf = O.synth_d(cfg, m, rf=True)
    steps = [1e-4, 1e-2, 1e-5, 1e-7, 1e-6, 1e-4, 1e-4, 1e-7, 1e-7]
    tol = [1e-8, 2e-3, 2e-3, 2e-3, 2e-3, 1e-7, 1e-7, 1e-8, 1e-8]
    for p in range(9):
        mp, mm = m.copy(), m.copy()
        mp[p] += steps[p]
        mm[p] -= steps[p]
        fd = (O.synth_d(cfg, mp) - O.synth_d(cfg, mm)) / (2 * steps[p])
        for s in range(4):
            if p == 6 and s in (0, 3):      # I and V do not depend on the azimuth
                assert np.abs(rf[s, p]).max() == 0.0
                continue
            scale = np.abs(fd[s]).max()
            if scale == 0:
                continue
            assert np.abs(fd[s] - rf[s, p]).max() / scale < tol[p], (p, s)


def test_rf_reference_magneto_optical_factor():
    """The reference differentiates F where the synthesis uses 2F
    (me_der.cu:71-74 vs mil_sinrf.cu:326): with scale 1 the B/vlos/dopp/damping
    RFs differ from the true derivative; eta0, gamma, S0, S1 do not."""
    g, cfg, _ = kat_cfg()
    m = g["model"].copy()
    _, rf1 = O.synth_d(cfg, m, rf=True)
    O.lib().orc_set_mo_scale(2.0)
    try:
        _, rf2 = O.synth_d(cfg, m, rf=True)
    finally:
        O.lib().orc_set_mo_scale(1.0)
    for p in (0, 5, 7, 8):
        np.testing.assert_array_equal(rf1[:, p], rf2[:, p])
    for p in (1, 2, 3, 4):
        assert np.abs(rf1[:, p] - rf2[:, p]).max() > 1e-3 * np.abs(rf2[:, p]).max()


def test_faithful_vs_fp64_synthesis():
    """The reference's own FP32 arithmetic stays within 2e-6 of FP64 in units
    of the intensity (per-row relative error can be large where Q, U vanish)."""
    rng = np.random.default_rng(5)
    l0, z = H.fe_line()
    lam, _ = H.grid()
    cfg = O.make_cfg(lam, l0, z, psf=O.psf_gauss(100.0, lam))
    for m in H.truth_models(50, rng):
        a = O.synth_f(cfg, m)
        b = O.synth_d(cfg, m)
        assert H.rel_to_I(a, b).max() < 2e-6


def test_svdcordic_is_a_similarity_transform():
    """18 parallel Jacobi steps: V orthogonal, w = diag(V^T A V), trace kept."""
    rng = np.random.default_rng(7)
    for _ in range(10):
        x = rng.normal(size=(10, 10))
        a = x @ x.T + np.diag(rng.uniform(0.1, 10, 10))
        w, v = O.svdcordic_d(a)
        np.testing.assert_allclose(v.T @ v, np.eye(10), atol=1e-12)
        np.testing.assert_allclose(np.diag(v.T @ a @ v), w, rtol=1e-10, atol=1e-10)
        assert w.sum() == pytest.approx(np.trace(a), rel=1e-12)
        # two sweeps reduce, but do not remove, the off-diagonal part
        off = v.T @ a @ v - np.diag(w)
        off0 = a - np.diag(np.diag(a))
        assert 0 < np.linalg.norm(off) < 0.5 * np.linalg.norm(off0)


def test_svdcordic_permutation_has_order_nine():
    perm = [0, 2, 4, 1, 6, 3, 8, 5, 9, 7]
    x = list(range(10))
    for k in range(1, 19):
        x = [perm[i] for i in x]
        assert (x == list(range(10))) == (k % 9 == 0)


def test_svdcordic_diagonal_input():
    a = np.diag(np.arange(1.0, 11.0))
    w, v = O.svdcordic_d(a)
    assert sorted(w) == pytest.approx(list(range(1, 11)))


def test_solve_drops_null_directions():
    """Rows and columns of fixed parameters are zero; the pseudo-inverse cut
    (|w| <= 1e-12) leaves their step at exactly zero (milosUtils.cu:350-353)."""
    rng = np.random.default_rng(11)
    x = rng.normal(size=(10, 10)).astype(np.float32)
    a = x @ x.T + 5 * np.eye(10, dtype=np.float32)
    a[9, :] = 0
    a[:, 9] = 0
    b = rng.normal(size=10).astype(np.float32)
    b[9] = 0
    d = O.solve_f(a, b)
    assert d[9] == 0.0


def test_svdcmp_reconstructs():
    rng = np.random.default_rng(13)
    a = rng.normal(size=(11, 11))
    u, w, v = O.svdcmp(a.copy())
    np.testing.assert_allclose(u @ np.diag(w) @ v.T, a, atol=1e-10)


def test_classical_estimates_recover_field():
    """Weak-field estimates on noiseless profiles: sign and size of B_los."""
    l0, z = H.fe_line()
    lam, _ = H.grid()
    cfg = O.make_cfg(lam, l0, z)
    for B, gm, vlos in ((500.0, 30.0, 0.5), (800.0, 150.0, -1.0)):
        m = np.array([10.0, B, vlos, 0.03, 0.1, gm, 45.0, 0.2, 0.8, 0.0, 1.0])
        obs = O.synth_f(cfg, m)
        est = O.classical(cfg, obs, model=np.array(H.GUESS), for_init=0)
        blos = est[7]
        assert np.sign(blos) == np.sign(np.cos(np.radians(gm)))
        assert abs(blos - B * np.cos(np.radians(gm))) < 0.2 * B
        # the centre-of-gravity velocity is biased low but has the right sign
        assert np.sign(est[2]) == np.sign(vlos) and abs(est[2]) < abs(vlos)
        assert abs(est[5] - gm) < 10


@pytest.mark.parametrize("nthreads", [1, 4])
def test_lm_recovers_truth(nthreads):
    """Faithful-mode inversion of noisy synthetic pixels reaches chi2 ~ 1."""
    rng = np.random.default_rng(17)
    l0, z = H.fe_line()
    lam, _ = H.grid()
    cfg = O.make_cfg(lam, l0, z, init=H.GUESS)
    t = H.truth_models(64, rng)
    obs = H.observations(cfg, t, rng)
    m, chi, it, acc, fit = O.lm_batch_f(cfg, obs, nthreads=nthreads)
    assert np.median(chi) < 1.5
    good = np.abs(m[:, 1] - t[:, 1]) < 50
    assert good.mean() > 0.8
    assert (it >= acc).all() and (it <= 50).all()


def test_lm_single_equals_batch():
    rng = np.random.default_rng(19)
    l0, z = H.fe_line()
    lam, _ = H.grid()
    cfg = O.make_cfg(lam, l0, z, init=H.GUESS)
    t = H.truth_models(4, rng)
    obs = H.observations(cfg, t, rng)
    mb, cb, ib, ab, fb = O.lm_batch_f(cfg, obs, nthreads=2)
    for p in range(4):
        m, c, i, a, f = O.lm_f(cfg, obs[p])
        np.testing.assert_array_equal(m, mb[p])
        assert c == cb[p] and i == ib[p] and a == ab[p]
        np.testing.assert_array_equal(f, fb[p])


def test_early_stop_rule():
    """stop_dchi2 > 0 (the ragged-batch option, not in the reference) ends a
    pixel at the first accepted step that improves chi2 by less than the
    threshold: it never lengthens a fit, a pixel it does not cut follows the
    reference trajectory exactly, and a threshold of 0 is the reference."""
    rng = np.random.default_rng(29)
    l0, z = H.fe_line()
    lam, _ = H.grid()
    t = H.truth_models(64, rng)
    base = O.make_cfg(lam, l0, z, init=H.GUESS)
    obs = H.observations(base, t, rng)
    m0, c0, i0, a0, _ = O.lm_batch_f(base, obs, nthreads=0)
    mz, cz, iz, az, _ = O.lm_batch_f(O.make_cfg(lam, l0, z, init=H.GUESS, stop_dchi2=0.0), obs, nthreads=0)
    np.testing.assert_array_equal(mz, m0)
    np.testing.assert_array_equal(iz, i0)
    me, ce, ie, ae, _ = O.lm_batch_f(O.make_cfg(lam, l0, z, init=H.GUESS, stop_dchi2=1e-4), obs, nthreads=0)
    assert (ie <= i0).all()
    cut = ie < i0
    assert cut.mean() > 0.5, cut.mean()
    np.testing.assert_array_equal(me[~cut], m0[~cut])
    # a cut fit ends on an accepted step
    assert (ae[cut] >= 1).all() and (ae[cut] <= a0[cut]).all()


def test_lm_step_decreases_chi2_with_large_damping():
    rng = np.random.default_rng(23)
    l0, z = H.fe_line()
    lam, _ = H.grid()
    cfg = O.make_cfg(lam, l0, z)
    t = H.truth_models(8, rng)
    obs = H.observations(cfg, t, rng)
    ok = 0
    for p in range(8):
        m0 = t[p].copy()
        m0[1] *= 1.05
        m0[2] += 0.05
        d, trial, c1, c0 = O.lm_step_f(cfg, m0, obs[p], 10.0)
        ok += c1 < c0
    assert ok >= 6


def test_stray_light_mixing():
    l0, z = H.fe_line()
    lam, _ = H.grid()
    cfg = O.make_cfg(lam, l0, z, fix=(1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1))
    sl = H.stray_profile(cfg)
    m = np.array([10.0, 1000, 0.5, 0.03, 0.1, 60, 30, 0.2, 0.8, 0, 0.7])
    pure = O.synth_f(cfg, m)
    mixed, rf = O.synth_f(cfg, m, slight=sl, rf=True)
    np.testing.assert_allclose(mixed, 0.7 * pure + 0.3 * sl, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(rf[:, 9], pure - sl, rtol=1e-6, atol=1e-7)
