"""CPU check of the algebra the FFT Poisson kernels (csrc/dct_fft.cu) are built
on: Makhoul's DCT-II through a complex FFT, the DCT-III through the inverse,
the sine transforms as (-1)^j times a DCT-III of the reversed sequence, two
real sequences per complex FFT, and the three passes with the packing the
kernels use (E-branch columns together, cosine-branch columns together).
Restated in numpy float64 (np.fft stands in for the shared-memory FFT) and
compared with the FP64 dense oracle, FFT_2D::doFFT's sums
(FFT/fft.cpp:191-284).  A second test replays the kernels' bit-reversed,
stage-paired radix-2 index arithmetic against np.fft.  The CUDA kernels
themselves are compared with the oracle in tests/test_gpu_dct_fft.py."""
import numpy as np
import pytest

from oracle import oracle as O


def _makhoul_perm(n):
    j = np.arange(n)
    return np.where(j & 1, n - 1 - (j >> 1), j >> 1)


def _dct2_pair(xa, xb):
    """DCT-II of the rows of xa and xb (real, [..., n]) by one complex FFT."""
    n = xa.shape[-1]
    v = np.empty(xa.shape, complex)
    v[..., _makhoul_perm(n)] = xa + 1j * xb  # v[m(j)] = x[j]
    z = np.fft.fft(v, axis=-1)
    zm = z[..., (-np.arange(n)) % n]
    va, vb = (z + np.conj(zm)) / 2, (z - np.conj(zm)) / 2j
    w = np.exp(-1j * np.pi * np.arange(n) / (2 * n))
    return (va * w).real, (vb * w).real


def _dct3_spec(x):
    """The Hermitian spectrum whose unnormalised IFFT gives C^T x (Makhoul order)."""
    n = x.shape[-1]
    xr = np.zeros_like(x)
    xr[..., 1:] = x[..., :0:-1]  # x[n-k], 0 at k = 0
    xd = x.copy()
    xd[..., 0] *= 2
    return 0.5 * (xd - 1j * xr) * np.exp(1j * np.pi * np.arange(n) / (2 * n))


def _dct3_pair(xa, xb):
    n = xa.shape[-1]
    z = np.fft.ifft(_dct3_spec(xa) + 1j * _dct3_spec(xb), axis=-1) * n
    z = z[..., _makhoul_perm(n)]  # y[j] = z[m(j)]
    return z.real, z.imag


def _sine_input(x):
    """b with S^T x = (-1)^j C^T b: b[0] = 0, b[k] = x[n-k]."""
    b = np.zeros_like(x)
    b[..., 1:] = x[..., :0:-1]
    return b


def fft_poisson(rho, step_x, step_y):
    nx, ny = rho.shape
    wx = np.pi * np.arange(nx) / nx
    wy = np.pi * np.arange(ny) / ny * (step_y / step_x)
    h = np.outer(np.where(np.arange(nx) == 0, 0.5, 1.0), np.where(np.arange(ny) == 0, 0.5, 1.0))
    den = wx[:, None] ** 2 + wy[None, :] ** 2
    den[0, 0] = 1.0
    K = 4.0 / nx / ny * h / den
    K[0, 0] = 0.0
    # pass 1: rows along y, two rows per complex FFT
    ta, tb = _dct2_pair(rho[0::2], rho[1::2])
    T = np.empty_like(rho)
    T[0::2], T[1::2] = ta, tb
    # pass 2: columns along x (transpose: columns become rows here)
    ca, cb = _dct2_pair(T.T[0::2], T.T[1::2])
    P = np.empty((ny, nx))
    P[0::2], P[1::2] = ca, cb
    P *= K.T
    sg_x = np.where(np.arange(nx) & 1, -1.0, 1.0)
    e = _sine_input(P * wx[None, :])
    x1a, x1b = _dct3_pair(e[0::2], e[1::2])  # E branch, two columns per IFFT
    x2a, x2b = _dct3_pair(P[0::2], P[1::2])  # cosine branch, two columns per IFFT
    X1 = np.empty((ny, nx))
    X2 = np.empty((ny, nx))
    X1[0::2], X1[1::2] = x1a * sg_x, x1b * sg_x
    X2[0::2], X2[1::2] = x2a, x2b
    X1, X2 = X1.T, X2.T
    # pass 3: rows along y; E_x and E_y in one IFFT, phi in another
    sg_y = np.where(np.arange(ny) & 1, -1.0, 1.0)
    ex, ey = _dct3_pair(X1, _sine_input(X2 * wy[None, :]))
    phi, _ = _dct3_pair(X2, np.zeros_like(X2))
    return ex, ey * sg_y, phi


@pytest.mark.parametrize("nx,ny,sy", [(8, 8, 1.0), (16, 64, 1.3), (64, 32, 0.7), (256, 256, 1.0)])
def test_fft_factorization_matches_dense_oracle(nx, ny, sy):
    rng = np.random.default_rng(nx * 7 + ny)
    rho = 1.0 + 0.3 * rng.standard_normal((nx, ny))
    sy = float(np.float32(sy))  # bin steps are float in the engine and the oracle
    ex, ey, phi = fft_poisson(rho, 1.0, sy)
    rx, ry, rp = O.poisson(rho, 1.0, sy)
    scale = max(np.abs(rx).max(), np.abs(ry).max())
    assert max(np.abs(ex - rx).max(), np.abs(ey - ry).max()) / scale < 1e-11
    assert np.abs(phi - rp).max() / np.abs(rp).max() < 1e-11


def _brev(i, logn):
    return int(format(i, f"0{logn}b")[::-1], 2)


def _stage_paired_fft(buf, logn, nseq, inverse):
    """block_fft's index arithmetic: an optional radix-2 stage 0 (odd log2 n),
    then stages s, s+1 applied together on the four elements i0 + {0,h,2h,3h};
    every element is touched exactly once per pass."""
    n, quarter = 1 << logn, 1 << (logn - 2)
    tw = np.concatenate([np.exp(-1j * np.pi * np.arange(h) / h) for h in (1 << s for s in range(logn))])
    tw = np.conj(tw) if inverse else tw
    first = logn & 1
    if first:
        for j in range(nseq * n // 2):
            a, c = buf[2 * j], buf[2 * j + 1]
            buf[2 * j], buf[2 * j + 1] = a + c, a - c
    for s in range(first, logn, 2):
        h = 1 << s
        seen = np.zeros(nseq * n, int)
        for j in range(nseq * quarter):
            q, b = j >> (logn - 2), j & (quarter - 1)
            pos = b & (h - 1)
            i0 = (q << logn) + ((b >> s) << (s + 2)) + pos
            idx = [i0, i0 + h, i0 + 2 * h, i0 + 3 * h]
            seen[idx] += 1
            a0, a1, a2, a3 = buf[idx]
            w1 = tw[h - 1 + pos]
            a0, a1 = a0 + a1 * w1, a0 - a1 * w1
            a2, a3 = a2 + a3 * w1, a2 - a3 * w1
            t2, t3 = a2 * tw[2 * h - 1 + pos], a3 * tw[2 * h - 1 + pos + h]
            buf[idx] = [a0 + t2, a1 + t3, a0 - t2, a1 - t3]
        assert (seen == 1).all()


@pytest.mark.parametrize("logn", [3, 4, 5, 6, 7])
@pytest.mark.parametrize("inverse", [False, True])
def test_stage_paired_index_arithmetic(logn, inverse):
    n, nseq = 1 << logn, 3
    rng = np.random.default_rng(logn)
    x = rng.standard_normal((nseq, n)) + 1j * rng.standard_normal((nseq, n))
    buf = np.zeros(nseq * n, complex)
    for q in range(nseq):
        for i in range(n):
            buf[q * n + _brev(i, logn)] = x[q, i]
    _stage_paired_fft(buf, logn, nseq, inverse)
    ref = np.fft.ifft(x, axis=1) * n if inverse else np.fft.fft(x, axis=1)
    assert np.abs(buf.reshape(nseq, n) - ref).max() < 1e-12 * np.abs(ref).max()
