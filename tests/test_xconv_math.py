"""Index arithmetic of the two-stage X pass (csrc/bdda_xconv.cuh), restated in
NumPy on the CPU: the 192-point axis as 24 x 8 (stage 1 DFT-24 over rows
j + 8q with twiddles w^(jk), middle DFT-8 over the rows of (j, k), Green
multiply at frequency k + 24 k2), with the Green's spectrum read from the
plan's digit-reversed storage through plan_position, gives the X pass's
convolution: the cropped output of an unnormalised inverse FFT of G(f) X(f)."""
import numpy as np

from bdda_b200 import _lib

M, A, B = 192, 24, 8


def plan_position(f, p):
    """The kernel's position of frequency f under the plan's DIF digit reversal."""
    d0 = f % p[0]
    d1 = (f // p[0]) % p[1]
    d2 = f // (p[0] * p[1])
    return d0 * (M // p[0]) + d1 * (M // (p[0] * p[1])) + d2


def digit_reversal(p):
    """Stored position -> frequency of a DIF transform with radices p (the plan's table)."""
    span = [M // p[0], M // (p[0] * p[1]), 1]
    rev = np.zeros(M, int)
    for k in range(M):
        rem, mult, f = k, 1, 0
        for s in range(3):
            q = rem // span[s]
            rem -= q * span[s]
            f += q * mult
            mult *= p[s]
        rev[k] = f
    return rev


def _plan_radices():
    import ctypes as C
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.bdda_plan_create((C.c_int * 3)(93, 112, 174), None, C.byref(h)) == 0
    try:
        r, ns = (C.c_int * 12)(), C.c_int()
        assert lib.bdda_plan_radices(h, 0, r, C.byref(ns)) == 0
        return [int(r[i]) for i in range(ns.value)]
    finally:
        lib.bdda_plan_destroy(h)


def test_plan_position_inverts_the_plans_digit_reversal():
    p = _plan_radices()
    assert p == [8, 8, 3]
    rev = digit_reversal(p)
    pos = np.array([plan_position(f, p) for f in range(M)])
    assert np.array_equal(np.sort(pos), np.arange(M))
    assert np.array_equal(rev[pos], np.arange(M))


def _gmul(g, v):
    gxx, gxy, gxz, gyy, gyz, gzz = g
    return np.array([gxx * v[0] + gxy * v[1] + gxz * v[2],
                     gxy * v[0] + gyy * v[1] + gyz * v[2],
                     gxz * v[0] + gyz * v[1] + gzz * v[2]])


def test_two_stage_split_gives_the_x_convolution():
    rng = np.random.default_rng(0)
    p = [8, 8, 3]
    n_in = n_out = 93
    x = np.zeros((3, M), complex)
    x[:, :n_in] = rng.standard_normal((3, n_in)) + 1j * rng.standard_normal((3, n_in))
    G = rng.standard_normal((M, 6)) + 1j * rng.standard_normal((M, 6))   # per frequency
    stored = np.zeros_like(G)
    stored[[plan_position(f, p) for f in range(M)]] = G                  # the plan's storage order
    X = np.fft.fft(x, axis=1)
    ref = np.fft.ifft(np.stack([_gmul(G[f], X[:, f]) for f in range(M)], 1), axis=1) * M
    w = np.exp(-2j * np.pi * np.arange(M) / M)
    for xl in (0, 1):   # both intermediate layouts: rows j + B k and j A + k
        row = (lambda j, k: j * A + k) if xl else (lambda j, k: j + B * k)
        tile = np.zeros((3, M), complex)
        for j in range(B):   # stage 1: rows at or past n_in are zero and not read
            v = np.array([x[:, j + B * q] if j + B * q < n_in else np.zeros(3) for q in range(A)]).T
            V = np.fft.fft(v, axis=1) * w[j * np.arange(A)]
            for k in range(A):
                tile[:, row(j, k)] = V[:, k]
        for k in range(A):   # middle: DFT-8, Green at frequency k + A k2, inverse DFT-8
            y = np.fft.fft(np.stack([tile[:, row(jj, k)] for jj in range(B)], 1), axis=1)
            for k2 in range(B):
                y[:, k2] = _gmul(stored[plan_position(k + A * k2, p)], y[:, k2])
            y = np.fft.ifft(y, axis=1) * B
            for jj in range(B):
                tile[:, row(jj, k)] = y[:, jj]
        out = np.zeros((3, M), complex)
        for j in range(B):   # stage 1 inverse: conjugate twiddles, inverse DFT-24
            v = np.stack([tile[:, row(j, k)] for k in range(A)], 1) * np.conj(w[j * np.arange(A)])
            V = np.fft.ifft(v, axis=1) * A
            for q in range(A):
                out[:, j + B * q] = V[:, q]
        err = np.max(np.abs(out[:, :n_out] - ref[:, :n_out])) / np.max(np.abs(ref))
        assert err < 1e-13, (xl, err)
