"""The offset symmetries the 3D Laplace M2L class kernels use to share one matrix per
symmetry class (laplace.cuh, kernels_trans.cu), checked on the CPU.

For the 16 isometries sigma = R^q C^s Z^t that keep the box lattice and the z axis
(R: quarter turn about z, C: y -> -y, Z: z -> -z), the M2L map of the offset sigma d
is T(sigma d) = Phi_out T(d) Phi_in, where Phi multiplies each stored coefficient
(n, m >= 0) by a power of i after an optional conjugation.  Here the singular
harmonics come from SciPy's associated Legendre functions (not the kernels'
recurrence), T from the M2L formula L_j^i = (-1)^j sum M_k^l S_{k+j}^{l+i}(d), and the
maps and the canonical offsets from their definitions; the kernels' one-byte form of
the maps (take the other entry of the coefficient, negate) is checked against them.
"""

import itertools
import math

import numpy as np
from scipy.special import lpmv


def _S(n, m, v):
    """S_n^m(v) = (n - m)! P_n^m(cos t) e^{i m p} / r^(n+1), no Condon-Shortley phase,
    S_n^{-m} = (-1)^m conj(S_n^m)."""
    am = abs(m)
    if am > n:
        return 0j
    x, y, z = v
    r = math.sqrt(x * x + y * y + z * z)
    p = (-1) ** am * lpmv(am, n, z / r)          # remove SciPy's (-1)^m
    val = math.factorial(n - am) * p * np.exp(1j * am * math.atan2(y, x)) / r ** (n + 1)
    return (-1) ** am * np.conj(val) if m < 0 else val


def _coeffs(p):
    return [(n, m) for n in range(p + 1) for m in range(n + 1)]


def _m2l(d, M, p):
    idx = _coeffs(p)
    full = {}
    for (n, m), v in zip(idx, M):
        full[(n, m)] = v
        if m > 0:
            full[(n, -m)] = (-1) ** m * np.conj(v)
    out = []
    for j, i in idx:
        s = sum(v * _S(k + j, l + i, d) for (k, l), v in full.items())
        out.append((-1) ** j * s)
    return np.array(out)


def _phi(M, p, code, out):
    q, s, t = code & 3, (code >> 2) & 1, (code >> 3) & 1
    res = []
    for (n, m), v in zip(_coeffs(p), M):
        e = 2 * t * (n + m) + (m * q if (out or not s) else -m * q)
        res.append(1j ** (e % 4) * (np.conj(v) if s else v))
    return np.array(res)


def _canonical(d):
    """(canonical offset, code) with d = R^q C^s Z^t (canonical offset)."""
    dx, dy, dz = d
    a, b = max(abs(dx), abs(dy)), min(abs(dx), abs(dy))
    for q, s in itertools.product(range(4), range(2)):
        x, y = a, (-b if s else b)
        for _ in range(q):
            x, y = -y, x
        if (x, y) == (dx, dy):
            return (a, b, abs(dz)), q | s << 2 | (8 if dz < 0 else 0)
    raise AssertionError(d)


def test_every_list2_offset_maps_to_its_canonical_matrix():
    p = 5
    rng = np.random.default_rng(0)
    idx = _coeffs(p)
    offsets = [d for d in itertools.product(range(-3, 4), repeat=3) if max(map(abs, d)) >= 2]
    assert len(offsets) == 316
    canon = set()
    for d in offsets:
        dc, code = _canonical(d)
        canon.add(dc)
        assert dc[0] >= dc[1] >= 0 and dc[2] >= 0
        M = rng.normal(size=len(idx)) + 1j * rng.normal(size=len(idx))
        M[[k for k, (n, m) in enumerate(idx) if m == 0]] = \
            M[[k for k, (n, m) in enumerate(idx) if m == 0]].real
        ref = _m2l(d, M, p)
        got = _phi(_m2l(dc, _phi(M, p, code, False), p), p, code, True)
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), (d, code)
    # canonical offsets a >= b >= 0, c >= 0 in [0, 3]: 10 (a, b) x 4 c, less the 6 with
    # every entry <= 1
    assert len(canon) == 34


def test_one_byte_form_of_the_maps():
    """The kernels' op bits (bit 0: take the other entry of the coefficient, bit 1:
    negate) against i^e conj^s for every phase, conjugation and entry."""
    def op(e, s, part):
        e &= 3
        if part == 0:
            neg = e == 2 or (e == 1 and not s) or (e == 3 and s)
        else:
            neg = e == 3 or (e == 0 and s) or (e == 2 and not s)
        return (e & 1) | int(neg) << 1

    a, b = 3.0, 5.0
    for e, s, part in itertools.product(range(4), range(2), range(2)):
        z = complex(a, -b if s else b) * 1j ** e
        want = (z.real, z.imag)[part]
        o = op(e, s, part)
        got = (a, b)[part ^ (o & 1)]
        assert (-got if o & 2 else got) == want, (e, s, part)
