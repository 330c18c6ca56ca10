"""CPU checks of the float32 roots of unity the FFT kernels use (``csrc/unit_consts.cuh``).

The header is generated by ``csrc/gen_unit_consts.py``; these tests check that the
committed header is what the generator writes, that every root is within rounding
of the exact value, and that the transforms built from them keep the wave's energy
(the nearest-rounded roots lose about 2.7e-8 per 16-point DFT, coherently).
"""

import cmath
import importlib.util
import math
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ptyrodactyl_b200", "csrc")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_unit_consts", os.path.join(CSRC, "gen_unit_consts.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _table(src, name):
    body = src[src.index(name + "(int r)"):]
    body = body[:body.index("default")]
    return {int(a): float(b) for a, b in re.findall(r"case (\d+): return ([0-9.e+-]+)f", body)}


@pytest.fixture(scope="module")
def tables():
    with open(os.path.join(CSRC, "unit_consts.cuh")) as f:
        src = f.read()
    return {n: _table(src, n) for n in ("bfly_m", "bfly_t", "unit_c", "unit_s")}


def test_header_matches_generator():
    pytest.importorskip("mpmath")
    gen = _gen()
    fsel, psel = gen.solve()
    with open(os.path.join(CSRC, "unit_consts.cuh")) as f:
        assert f.read() == gen.render(fsel, psel)


def _fact(t, k, direction):
    """Restatement of fact_tw<DIR>(k) in fft_core.cuh."""
    k &= 63
    q, r = k >> 4, k & 15
    m, tt, a = (t["bfly_m"][r], t["bfly_t"][r], True) if r <= 8 else (t["bfly_m"][16 - r], t["bfly_t"][16 - r], False)
    for _ in range(q):
        m, tt, a = (m, -tt, False) if a else (-m, -tt, True)
    if direction < 0:
        if a:
            tt = -tt
        else:
            m, tt = -m, -tt
    return m * (1 + 1j * tt) if a else m * (tt + 1j), a


def _w64(t, k, direction):
    """Restatement of w64<DIR>(k) in fft_core.cuh."""
    k &= 63
    q, r = k >> 4, k & 15
    c0, s0 = t["unit_c"][r], t["unit_s"][r]
    c, s = [(c0, s0), (-s0, c0), (-c0, -s0), (s0, -c0)][q]
    return complex(c, -s if direction < 0 else s)


@pytest.mark.parametrize("direction", [-1, 1])
def test_roots_within_rounding_and_forms_consistent(tables, direction):
    for k in range(64):
        if k % 16 == 0:
            continue
        exact = cmath.exp(direction * 2j * math.pi * k / 64)
        w, form_a = _fact(tables, k, direction)
        assert abs(w - exact) < 5e-8
        assert form_a == (abs(exact.real) >= abs(exact.imag))
        assert abs(_w64(tables, k, direction) - exact) < 5e-8


def test_transform_energy_bias_small(tables):
    gen = _gen()
    d = {r: math.hypot(1.0, tables["bfly_t"][r]) * tables["bfly_m"][r] - 1.0 for r in range(1, 9)}
    assert abs(sum(gen.dit_stage_biases(d, 16))) < 1e-9
    assert abs(sum(gen.dit_stage_biases(d, 32))) < 3e-9
    pd = {r: math.hypot(tables["unit_c"][r], tables["unit_s"][r]) - 1.0 for r in range(1, 16)}
    for n1, n2 in gen.SHAPES[2:]:
        w, n = gen.table_weights(n1, n2)
        assert abs(2 * sum(cnt * pd[r] for r, cnt in w.items()) / n) < 1e-9, (n1, n2)
