"""The oracle itself: pinned to the reference's golden vectors and known answers."""

import numpy as np
import pytest

from oracle import jax_prng
from oracle import multislice_ref as R
from tests.conftest import rel_l2


def test_threefry_known_answers():
    # Random123 known-answer vectors for Threefry-2x32-20
    cases = [((0, 0), (0, 0), (0x6B200159, 0x99BA4EFE)),
             ((0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF), (0x1CB996FC, 0xBB002BE7)),
             ((0x13198A2E, 0x03707344), (0x243F6A88, 0x85A308D3), (0xC4923A9C, 0x483DF7A0))]
    for key, ctr, want in cases:
        a, b = jax_prng.threefry2x32(key, np.array([ctr[0]], np.uint32), np.array([ctr[1]], np.uint32))
        assert (int(a[0]), int(b[0])) == want


def test_golden_input_regenerates(golden):
    pot = jax_prng.uniform_f64(jax_prng.prng_key(42), (32, 32, 2)) * 10.0
    assert np.array_equal(pot, golden["pot"])


def _golden_stem(golden, dtype=np.complex128):
    g = golden
    probe = R.make_probe(float(g["voltage_kv"]), float(g["aperture_mrad"]), (32, 32),
                         float(g["calib_ang"]) * 100.0)
    return R.stem_4d(g["pot"], float(g["slice_thickness_ang"]), float(g["calib_ang"]), probe[..., None],
                     [1.0], float(g["calib_ang"]), float(g["voltage_kv"]), g["positions_px"],
                     float(g["calib_ang"]), dtype=dtype)


def test_oracle_matches_reference_golden(golden):
    """plan01_ug_reference.npz (reference capture, float64)."""
    g = golden
    probe = R.make_probe(100.0, 20.0, (32, 32), 20.0)
    cbed = R.cbed_image(g["pot"], 2.0, 0.2, probe[..., None], [1.0], 0.2, 100.0)
    assert np.max(np.abs(cbed - g["cbed"])) < 1e-13
    s4 = _golden_stem(g)
    assert np.max(np.abs(s4["data"] - g["stem4d"])) < 1e-13
    assert s4["scan_positions"].shape == (4, 2)


def test_oracle_c64_close_to_c128(golden):
    s64 = _golden_stem(golden, np.complex64)["data"]
    assert rel_l2(s64, golden["stem4d"]) < 1e-5


def test_pattern_sum_is_aperture_count(golden):
    n_ap = R.aperture_count(100.0, 20.0, (32, 32), 20.0)
    assert n_ap == 37
    assert abs(golden["cbed"].sum() - 37.0) < 1e-9
    assert np.allclose(golden["stem4d"].sum(axis=(1, 2)), 37.0)


def test_wavelength_and_sigma_values():
    # values quoted for the reference's constants (types/constants.py:291-340)
    for kv, lam in ((60, 0.048661), (100, 0.037014), (200, 0.025079), (300, 0.019687)):
        assert abs(R.relativistic_wavelength_ang(kv) - lam) < 5e-7
    for kv, sig in ((100, 9.2440e-4), (200, 7.2884e-4), (300, 6.5262e-4)):
        assert abs(R.interaction_sigma(kv) - sig) / sig < 1e-4


def test_vjp_matches_finite_differences():
    rng = np.random.default_rng(5)
    n, s = 16, 3
    pot = rng.uniform(0, 30, (n, n, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 40.0, defocus_ang=-20.0)
    pos = np.array([[0.3, -0.4], [1.2, 0.7]])
    g = rng.normal(size=(2, n, n))

    def loss(v, beam):
        d = R.stem_4d(v, 1.5, 0.4, beam[..., None], [1.0], 0.4, 200.0, pos, 0.4)["data"]
        return float(np.sum(g * d))

    dv, dbeam = R.stem_4d_vjp(pot, 1.5, 0.4, probe[..., None], [1.0], 0.4, 200.0, pos, 0.4, g)
    for (y, x, k) in [(3, 4, 0), (8, 8, 1), (12, 2, 2)]:
        e = np.zeros_like(pot)
        e[y, x, k] = 1e-4
        fd = (loss(pot + e, probe) - loss(pot - e, probe)) / 2e-4
        assert abs(fd - dv[y, x, k]) <= 1e-6 * max(1.0, abs(fd))
    # complex beam gradient, JAX convention grad = dL/dRe - i dL/dIm
    for (y, x) in [(8, 8), (7, 9)]:
        e = np.zeros_like(probe)
        e[y, x] = 1e-5
        fre = (loss(pot, probe + e) - loss(pot, probe - e)) / 2e-5
        fim = (loss(pot, probe + 1j * e) - loss(pot, probe - 1j * e)) / 2e-5
        assert abs(dbeam[y, x, 0] - (fre - 1j * fim)) <= 1e-6 * max(1.0, abs(fre) + abs(fim))


def test_golden_gradient_is_null(golden):
    """grad of sum(cbed) w.r.t. V vanishes (the sum is the aperture count for any V)."""
    g = golden
    probe = R.make_probe(100.0, 20.0, (32, 32), 20.0)
    dv, _ = R.stem_4d_vjp(g["pot"], 2.0, 0.2, probe[..., None], [1.0], 0.2, 100.0, np.zeros((1, 2)), 0.2,
                          np.ones((1, 32, 32)))
    assert np.max(np.abs(dv)) < 1e-12
    assert np.max(np.abs(g["grad_pot"])) < 1e-12


def test_oracle_atom_backed_matches_reference_golden(golden):
    """stem4d_sharded of the golden capture (atom-backed slices, plan01_ug_capture.py:74-97)."""
    g = golden
    probe = R.make_probe(100.0, 20.0, (32, 32), 20.0)
    atoms = np.array([[2.0, 2.5, 0.25], [4.5, 5.0, 2.25], [3.0, 4.0, 1.25]])
    out = R.stem4d_sharded(probe[..., None], [1.0], atoms, [0, 0, 0], [[0.0, 2.0], [2.0, 4.0]],
                           g["pot"][..., 0][None], 100.0, 0.2, g["positions_px"] * 0.2)
    assert np.max(np.abs(out["data"] - g["stem4d_sharded"])) < 1e-13


def test_oracle_annular_detector_known_answer():
    """test_simulations.py:84-122: 0-1000 mrad covers every pixel of a 4x4 pattern."""
    data = np.arange(6 * 4 * 4, dtype=np.float64).reshape(6, 4, 4)
    img = R.annular_detector(data, 0.25, 80.0, 0.0, 1000.0, (2, 3))
    assert np.array_equal(img, np.array([[120.0, 376.0, 632.0], [888.0, 1144.0, 1400.0]]))


def test_oracle_annular_detector_golden_invariant(golden):
    """A detector covering the whole pattern collects the aperture count (37 per probe)."""
    g = golden
    fc = 1.0 / (32 * 0.2)
    full = R.annular_detector(g["stem4d"], fc, 100.0, 0.0, 1e6, (2, 2))
    assert np.allclose(full, 37.0, rtol=1e-12)
    bf = R.annular_detector(g["stem4d"], fc, 100.0, 0.0, 20.0, (2, 2))
    df = R.annular_detector(g["stem4d"], fc, 100.0, 20.0 + 1e-9, 1e6, (2, 2))
    assert np.allclose(bf + df, full, rtol=1e-12)


def test_product_mask_matches_oracle_mask():
    from ptyrodactyl_b200.detectors import annular_mask
    for n, fc, kv, a, b in [(64, 0.05, 200.0, 10.0, 40.0), (128, 0.03, 300.0, 0.0, 25.0), (16, 0.2, 80.0, 5.0, 5.0)]:
        assert np.array_equal(annular_mask((n, n), fc, kv, a, b), R.annular_mask((n, n), fc, kv, a, b))


def _jvp_case(seed=9, n=16, s=3, m=2):
    rng = np.random.default_rng(seed)
    pot = rng.uniform(0, 30, (n, n, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 40.0, defocus_ang=-20.0)
    beam = np.stack([probe * np.exp(0.3j * k) * (1.0 - 0.3 * k) for k in range(m)], axis=-1)
    w = np.linspace(1.0, 0.5, m)
    w = w / w.sum()
    pos = np.array([[0.3, -0.4], [1.2, 0.7]])
    dv = rng.normal(size=pot.shape)
    db = (rng.normal(size=beam.shape) + 1j * rng.normal(size=beam.shape)) * 0.01
    return pot, beam, w, pos, dv, db


def test_oracle_jvp_matches_finite_differences():
    pot, beam, w, pos, dv, db = _jvp_case()
    args = (1.5, 0.4)

    def f(v, b):
        return R.stem_4d(v, 1.5, 0.4, b, w, 0.4, 200.0, pos, 0.4)["data"]

    data, dd = R.stem_4d_jvp(pot, *args, beam, w, 0.4, 200.0, pos, 0.4, dslices=dv, dbeam=db)
    assert np.allclose(data, f(pot, beam), rtol=1e-12, atol=1e-14)
    eps = 1e-5
    fd = (f(pot + eps * dv, beam + eps * db) - f(pot - eps * dv, beam - eps * db)) / (2 * eps)
    assert np.max(np.abs(fd - dd)) <= 1e-6 * np.max(np.abs(dd))


def test_oracle_jvp_is_the_transpose_of_the_vjp():
    """<J v, g> = <dV, vV> + Re sum(dbeam_jax * vbeam) (dot-product test)."""
    pot, beam, w, pos, dv, db = _jvp_case(seed=4)
    g = np.random.default_rng(1).normal(size=(2, 16, 16))
    _, dd = R.stem_4d_jvp(pot, 1.5, 0.4, beam, w, 0.4, 200.0, pos, 0.4, dslices=dv, dbeam=db)
    gv, gb = R.stem_4d_vjp(pot, 1.5, 0.4, beam, w, 0.4, 200.0, pos, 0.4, g)
    lhs = np.sum(dd * g)
    rhs = np.sum(gv * dv) + np.real(np.sum(gb * db))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_oracle_ensemble_reduces_to_plain_and_explicit_composition():
    """Zero-width ensembles give the plain CBED; a jitter axis equals the weighted
    sum of CBEDs of explicitly shifted beams (test_simulations.py:243-285)."""
    rng = np.random.default_rng(0)
    n = 16
    pot = rng.uniform(0, 20, (n, n, 2))
    probe = R.make_probe(200.0, 25.0, (n, n), 20.0)
    modes = np.stack([probe, np.roll(probe, 1, 0)], -1)
    w = np.array([0.7, 0.3])
    axes = [(np.arange(2.0)[:, None], w, "incoherent", "probe_modes"), R.jitter_axis(0.0, 2),
            R.coherence_axis(0.0, 0.0, 2)]
    plain = R.cbed_image(pot, 1.5, 0.2, modes, w, 0.2, 200.0)
    assert np.max(np.abs(R.ensemble_cbed(pot, 1.5, 0.2, modes, 0.2, 200.0, axes) - plain)) < 1e-13
    jit = R.jitter_axis(0.15, 2)
    e = R.ensemble_cbed(pot, 1.5, 0.2, probe[..., None], 0.2, 200.0, [jit])
    explicit = sum(wk * R.cbed_image(pot, 1.5, 0.2, R.shift_beam_fourier(probe[..., None], d[None], 0.2)[0], [1.0],
                                     0.2, 200.0) for d, wk in zip(jit[0], jit[1]))
    assert np.max(np.abs(e - explicit)) < 1e-13
    # Gauss-Hermite(2) nodes are +-sigma with weight 1/4 per (dy, dx) pair
    assert np.allclose(np.abs(jit[0]), 0.15) and np.allclose(jit[1], 0.25)


def test_product_producers_match_oracle():
    from ptyrodactyl_b200 import ensemble as E
    for q in (1, 2, 3):
        d = E.position_jitter_to_distribution(0.2, q)
        s, w, _, _ = R.jitter_axis(0.2, q)
        assert np.allclose(d.samples.numpy(), s) and np.allclose(d.weights.numpy(), w)
        c = E.coherence_to_distribution(0.7, 0.05, q)
        s, w, _, _ = R.coherence_axis(0.7, 0.05, q)
        assert np.allclose(c.samples.numpy(), s) and np.allclose(c.weights.numpy(), w)
    with pytest.raises(ValueError, match="n_quad must be positive"):
        E.position_jitter_to_distribution(0.2, 0)
    with pytest.raises(ValueError, match="sigma_ang must be non-negative"):
        E.position_jitter_to_distribution(-0.2, 2)


def test_ensemble_axis_validation():
    import ptyrodactyl_b200 as pb
    jit = pb.position_jitter_to_distribution(0.1, 2)
    with pytest.raises(ValueError, match="coherence.samples must have width 3"):
        pb.create_ensemble_axes(coherence=jit)
    with pytest.raises(ValueError, match="samples and weights must share leading dimension"):
        pb.create_distribution(np.zeros((3, 1)), np.ones(2))
    with pytest.raises(ValueError, match="weights must be non-negative"):
        pb.create_distribution(np.zeros((2, 1)), [1.0, -1.0])
    ax = pb.create_ensemble_axes(position_jitter=jit)
    beam = pb.create_probe_modes(np.ones((16, 16, 2), np.complex64), [0.5, 0.5], 0.2)
    from ptyrodactyl_b200.ensemble import _axis_maps, ensemble_axes_for_cbed
    axes = ensemble_axes_for_cbed(ax, beam)
    assert [a.axis_id for a in axes] == ["probe_modes", "position_jitter"]
    with pytest.raises(ValueError, match="multimode probes require a first probe_modes axis"):
        _axis_maps((jit,), 2)


def test_oracle_resize_weights_properties():
    """Upscaling by 2 interpolates at quarter offsets; downscaling by 2 widens the
    triangle to four taps (antialias), renormalised at the edges; rows sum to one."""
    w = R.resize_linear_weights(4, 8)
    assert np.allclose(w.sum(axis=0), 1.0)
    x = np.arange(4.0)
    assert np.allclose((w.T @ x)[1:-1], [0.25, 0.75, 1.25, 1.75, 2.25, 2.75])
    d = R.resize_linear_weights(8, 4)
    assert np.allclose(d.sum(axis=0), 1.0)
    assert np.allclose(d[:, 1], [0.0, 0.125, 0.375, 0.375, 0.125, 0.0, 0.0, 0.0])  # interior taps
    assert np.allclose(d.T @ np.arange(8.0), [5 / 7, 2.5, 4.5, 44 / 7])  # edges renormalised
    from ptyrodactyl_b200.detectors import linear_resize_weights
    for a, b in [(4, 8), (8, 4), (100, 37), (37, 64), (64, 64)]:
        assert np.allclose(linear_resize_weights(a, b), R.resize_linear_weights(a, b).T)


def test_oracle_position_gradient_matches_finite_differences():
    rng = np.random.default_rng(6)
    n, s = 16, 3
    pot = rng.uniform(0, 30, (n, n, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 40.0, defocus_ang=-20.0)
    modes = np.stack([probe, np.roll(probe, 1, 0) * 0.5j], -1)
    w = [0.7, 0.3]
    pos = np.array([[0.3, -0.4], [1.2, 0.7]])
    g = rng.normal(size=(2, n, n))

    def loss(p):
        return float(np.sum(g * R.stem_4d(pot, 1.5, 0.4, modes, w, 0.4, 200.0, p, 0.4)["data"]))

    _, _, dpos = R.stem_4d_vjp(pot, 1.5, 0.4, modes, w, 0.4, 200.0, pos, 0.4, g, with_positions=True)
    for i in range(2):
        for c in range(2):
            e = np.zeros_like(pos)
            e[i, c] = 1e-5
            fd = (loss(pos + e) - loss(pos - e)) / 2e-5
            assert abs(fd - dpos[i, c]) <= 1e-6 * max(1.0, abs(fd))


@pytest.mark.parametrize("z,expected_sum,expected_max", [(6, 3304.630500664369, 599.0660669230273),
                                                         (14, 7467.50633667953, 1309.8209272295387),
                                                         (79, 16835.066119859865, 6296.83419348897)])
def test_oracle_single_atom_potential_matches_captured_reference(z, expected_sum, expected_max):
    """The reference's captured Kirkland C/Si/Au values (test_atom_potentials.py:31-63,
    rtol 2e-15 there): the oracle restates the reference's Bessel approximations."""
    pot = R.single_atom_potential(z, 0.2, (16, 16), supersampling=2, parameterization="kirkland")
    assert abs(pot.sum() - expected_sum) <= 2e-15 * expected_sum
    assert abs(pot.max() - expected_max) <= 2e-15 * expected_max
