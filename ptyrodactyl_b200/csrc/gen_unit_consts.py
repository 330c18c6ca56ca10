"""Generate ``unit_consts.cuh``: the float32 roots of unity W_64^r used by the FFT kernels.

Run ``python ptyrodactyl_b200/csrc/gen_unit_consts.py`` to rewrite the header; the
CPU test ``tests/test_unit_consts.py`` checks that the committed header matches.

Why the constants are not simply cos/sin rounded to nearest: every multiply by a
rounded root of unity w' = (1 + d) w scales the energy of the value it touches by
(1 + d)^2. The roots exp(2 pi i r / 64) that the radix-2 stages and the four-step
twiddle tables use happen to round to magnitudes below one for most r
(d = -2.9e-8, -2.9e-8, -1.7e-8 for r = 2, 4, 8), so a 256-point transform loses
about 5e-8 of the wave's energy, coherently, every time it runs; over the 200
one-dimensional transforms of a 50-slice multislice run that is a 1e-5 loss of
pattern intensity, while the physics conserves it exactly (|T| = 1, the
propagator is unitary).

Each constant here is instead picked among the float32 neighbours of the exact
value whose phase error stays within PHASE_LIMIT (about 0.75 ulp), so that the
expected energy change of every transform the kernels run is close to zero:

* ``bfly_m/bfly_t`` (r = 0..8): the factored butterfly twiddle
  w = M (1 + i T) (|cos| >= |sin|; r > 8 uses the swapped pair of 16 - r), so its
  magnitude is M sqrt(1 + T^2). A radix-2 stage that multiplies half its inputs
  by roots of magnitude 1 + d_k changes the energy of spread-out data by the mean
  of d_k over its butterflies, so the constants are chosen to make the sum of
  those stage means small for the 8-, 16- and 32-point DFTs.
* ``unit_c/unit_s`` (r = 0..15): cos and sin of 2 pi r / 64 for plain complex
  multiplies (the 512-point half-line stage and the four-step twiddle tables,
  whose entries at multiples of N/64 are taken from this table), chosen so the
  mean magnitude error over each table the kernels build (N = 64..1024) and over
  the half-line stage is close to zero.

A penalty on each constant's own magnitude error keeps any single constant from
carrying a large error that another cancels.
"""

from __future__ import annotations

import os
import sys

import numpy as np

try:
    import mpmath as mp
except ImportError:  # pragma: no cover - mpmath ships with the image's sympy
    mp = None

PHASE_LIMIT = 4.5e-8  # rad; round-to-nearest of a unit-magnitude pair gives up to ~4.2e-8
MAG_LIMIT = 3.0e-8  # no constant's own magnitude error exceeds that of nearest rounding
SPAN = 3  # float32 neighbours searched on each side of the nearest value
PENALTY = 0.05  # weight of each constant's own |magnitude error| in the objective
# (N1, N2) of the line transforms (N = N1 N2) whose four-step tables are built
SHAPES = [(4, 4), (4, 8), (8, 8), (8, 16), (16, 16), (16, 32), (32, 32)]
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "unit_consts.cuh")


def _neighbours(x: float, k: int):
    v = np.float32(x)
    out, up, dn = [v], v, v
    for _ in range(k):
        up = np.nextafter(up, np.float32(np.inf))
        dn = np.nextafter(dn, np.float32(-np.inf))
        out += [up, dn]
    return [float(o) for o in out]


def _angle(r: int):
    return 2 * mp.pi * r / 64


def _fact_candidates(r: int):
    """(magnitude error, phase error, M, T) with M (1 + i T) ~ exp(i 2 pi r / 64), r <= 8."""
    phi = _angle(r)
    out = []
    for m in _neighbours(float(mp.cos(phi)), SPAN):
        for t in _neighbours(float(mp.tan(phi)), SPAN):
            mag = float(mp.mpf(m) * mp.sqrt(1 + mp.mpf(t) ** 2) - 1)
            ph = float(mp.atan(mp.mpf(t)) - phi)
            if abs(ph) <= PHASE_LIMIT and abs(mag) <= MAG_LIMIT:
                out.append((mag, ph, m, t))
    return sorted(out, key=lambda c: abs(c[0]) + abs(c[1]))


def _plain_candidates(r: int):
    """(magnitude error, phase error, c, s) with c + i s ~ exp(i 2 pi r / 64)."""
    phi = _angle(r)
    out = []
    for c in _neighbours(float(mp.cos(phi)), SPAN):
        for s in _neighbours(float(mp.sin(phi)), SPAN):
            mag = float(mp.sqrt(mp.mpf(c) ** 2 + mp.mpf(s) ** 2) - 1)
            ph = float(mp.atan2(mp.mpf(s), mp.mpf(c)) - phi)
            if abs(ph) <= PHASE_LIMIT and abs(mag) <= MAG_LIMIT:
                out.append((mag, ph, c, s))
    return sorted(out, key=lambda c: abs(c[0]) + abs(c[1]))


def _fact_mag(d, r):
    """Magnitude error of the factored root for any r in 1..15 (r > 8 mirrors 16 - r)."""
    return d[r if r <= 8 else 16 - r]


def dit_stage_biases(d, radix: int):
    """Mean magnitude error of each radix-2 stage of a ``radix``-point DIT DFT; the
    stage of span HALF uses k = j * 64 / (2 HALF), j < HALF (exact for k % 16 == 0)."""
    out = []
    half = 1
    while 2 * half <= radix:
        ks = [j * (64 // (2 * half)) for j in range(half)]
        out.append(sum(0.0 if k % 16 == 0 else _fact_mag(d, k % 16) for k in ks) / half)
        half *= 2
    return out


def table_weights(n1: int, n2: int):
    """How often each 64th root (r = k mod 16, k = j 64 / N) occurs in the four-step
    table entries W_N^{t k2}, t < n1, k2 < n2, and the table's size."""
    n = n1 * n2
    w = {}
    for t in range(n1):
        for k2 in range(n2):
            j = (t * k2) % n
            if (j * 64) % n == 0:
                r = (j * 64 // n) % 16
                if r:
                    w[r] = w.get(r, 0) + 1
    return w, n


def _fact_cost(d):
    cost = 0.0
    for radix in (8, 16, 32):
        cost += abs(sum(dit_stage_biases(d, radix)))
    return cost + PENALTY * sum(abs(v) for v in d.values())


def _plain_cost(d):
    cost = 0.0
    for n1, n2 in SHAPES:
        w, n = table_weights(n1, n2)
        cost += abs(2 * sum(cnt * d[r] for r, cnt in w.items()) / n)
    # decimation-in-frequency first stage of the half-paired 512-point line: k = 2 j, j < 16
    cost += abs(sum(d[(2 * j) % 16] if (2 * j) % 16 else 0.0 for j in range(16)) / 16)
    return cost + PENALTY * sum(abs(v) for k, v in d.items() if k)


def _descend(cands, cost_of):
    """Coordinate descent from the most accurate candidates (deterministic; the plain
    table has too many constants for an exhaustive search)."""
    pick = {r: 0 for r in cands}

    def mags(p):
        return {r: cands[r][i][0] for r, i in p.items()}

    best = cost_of(mags(pick))
    for _ in range(50):
        improved = False
        for r in sorted(cands):
            for i in range(len(cands[r])):
                trial = dict(pick)
                trial[r] = i
                c = cost_of(mags(trial))
                if c < best - 1e-18:
                    best, pick, improved = c, trial, True
        if not improved:
            break
    return {r: cands[r][i] for r, i in pick.items()}, best


def solve():
    if mp is None:
        raise RuntimeError("mpmath is needed to generate the constants")
    mp.mp.dps = 40
    fact = {r: _fact_candidates(r) for r in range(1, 9)}
    # only r in {2, 4, 6, 8} is reachable from DFTs of at most 32 points; the others
    # keep their most accurate candidate
    fact_free = {r: fact[r] for r in (2, 4, 6, 8)}

    def fact_cost_full(dsub):
        d = {r: fact[r][0][0] for r in range(1, 9)}
        d.update(dsub)
        return _fact_cost(d)

    fpick, best = None, None
    for c2 in fact_free[2]:
        for c4 in fact_free[4]:
            for c6 in fact_free[6]:
                for c8 in fact_free[8]:
                    trial = {2: c2, 4: c4, 6: c6, 8: c8}
                    c = fact_cost_full({r: v[0] for r, v in trial.items()})
                    if best is None or c < best - 1e-18:
                        fpick, best = trial, c
    fsel = {r: fact[r][0] for r in range(1, 9)}
    fsel.update(fpick)
    plain = {r: _plain_candidates(r) for r in range(1, 16)}
    psel, _ = _descend(plain, lambda d: _plain_cost({0: 0.0, **d}))
    return fsel, psel


def _hex(x: float) -> str:
    return float(np.float32(x)).hex()


def render(fsel, psel) -> str:
    fd = {r: fsel[r][0] for r in range(1, 9)}
    pd = {0: 0.0, **{r: psel[r][0] for r in range(1, 16)}}
    lines = [
        "// Generated by gen_unit_consts.py; do not edit by hand.",
        "// float32 roots of unity W_64^r = exp(2 pi i r / 64) chosen among the neighbours",
        "// of the exact values (phase error <= %.1e rad) so that the expected energy" % PHASE_LIMIT,
        "// change of each transform built from them is close to zero.",
        "#pragma once",
        "",
        "namespace ptyro {",
        "",
        "// factored butterfly twiddle M (1 + i T) for r = 0..8 (r > 8 uses 16 - r swapped)",
        "__device__ __forceinline__ float bfly_m(int r) {",
        "  switch (r) {",
        "    case 0: return 1.0f;",
    ]
    for r in range(1, 9):
        lines.append("    case %d: return %sf;  // |w| - 1 = %+.2e, phase error %+.2e" %
                     (r, repr(float(np.float32(fsel[r][2]))), fsel[r][0], fsel[r][1]))
    lines += ["    default: return 0.0f;", "  }", "}", "",
              "__device__ __forceinline__ float bfly_t(int r) {", "  switch (r) {", "    case 0: return 0.0f;"]
    for r in range(1, 9):
        lines.append("    case %d: return %sf;" % (r, repr(float(np.float32(fsel[r][3])))))
    lines += ["    default: return 0.0f;", "  }", "}", "",
              "// cos and sin of 2 pi r / 64 for plain complex multiplies, r = 0..15",
              "__device__ __host__ __forceinline__ float unit_c(int r) {", "  switch (r) {", "    case 0: return 1.0f;"]
    for r in range(1, 16):
        lines.append("    case %d: return %sf;  // |w| - 1 = %+.2e, phase error %+.2e" %
                     (r, repr(float(np.float32(psel[r][2]))), psel[r][0], psel[r][1]))
    lines += ["    default: return 0.0f;", "  }", "}", "",
              "__device__ __host__ __forceinline__ float unit_s(int r) {", "  switch (r) {", "    case 0: return 0.0f;"]
    for r in range(1, 16):
        lines.append("    case %d: return %sf;" % (r, repr(float(np.float32(psel[r][3])))))
    lines += ["    default: return 0.0f;", "  }", "}", ""]
    # document the residual biases
    lines.append("// expected energy change per transform (spread-out data):")
    for radix in (8, 16, 32):
        lines.append("//   %2d-point DIT DFT: %+.2e" % (radix, sum(dit_stage_biases(fd, radix))))
    for n1, n2 in SHAPES:
        w, n = table_weights(n1, n2)
        lines.append("//   64th-root entries of the %4d-point four-step table: %+.2e" %
                     (n, 2 * sum(cnt * pd[r] for r, cnt in w.items()) / n))
    lines += ["", "}  // namespace ptyro", ""]
    return "\n".join(lines)


def main(argv):
    fsel, psel = solve()
    text = render(fsel, psel)
    if "--check" in argv:
        with open(OUT) as f:
            return 0 if f.read() == text else 1
    with open(OUT, "w") as f:
        f.write(text)
    print(text)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
