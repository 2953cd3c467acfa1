"""The geometry behind the catalogue's FFT convolution (model.cu,
cat_conv_forward / cat_conv_adjoint), checked with numpy on the CPU.

A batch draws each galaxy on a canvas padded by pw//2, ph//2 on each side
(drawing dw x dh); the brute-force kernels then compute, for the W x H
outputs,

    forward  out(x, y) = sum_{i<pw, j<ph} conv(x + i, y + j) psf(pw-1-i, ph-1-j)
    adjoint  g(U, V)   = sum_{i<pw, j<ph} w(U + 1 - pw + i, V + 1 - ph + j) psf(i, j)

(w zero outside the outputs).  The FFT form reads the first as the circular
convolution at offset (pw - 1, ph - 1) and the second as the circular
correlation of w placed at (pw - 1, ph - 1), on a grid of only the drawing's
size rounded up: nothing the forward reads wraps around, and what the adjoint
wraps lands on the zeros below that offset.  These tests assert exactly that,
for odd and even PSF sides and non-square shapes, on the smallest grid the
argument allows (the drawing itself)."""
import numpy as np
import pytest


def _brute_forward(conv, psf, W, H):
    ph, pw = psf.shape
    out = np.zeros((H, W))
    for j in range(ph):
        for i in range(pw):
            out += conv[j:j + H, i:i + W] * psf[ph - 1 - j, pw - 1 - i]
    return out


def _brute_adjoint(w, psf, dw, dh):
    ph, pw = psf.shape
    H, W = w.shape
    # w placed at (pw - 1, ph - 1) on a zero canvas large enough for every read
    big = np.zeros((dh + ph, dw + pw))
    big[ph - 1:ph - 1 + H, pw - 1:pw - 1 + W] = w
    g = np.zeros((dh, dw))
    for j in range(ph):
        for i in range(pw):
            g += big[j:j + dh, i:i + dw] * psf[j, i]
    return g


def _circ_forward(conv, psf, W, H, N, M):
    ph, pw = psf.shape
    a = np.zeros((M, N))
    a[:conv.shape[0], :conv.shape[1]] = conv
    k = np.zeros((M, N))
    k[:ph, :pw] = psf
    c = np.real(np.fft.ifft2(np.fft.fft2(a) * np.fft.fft2(k)))
    return c[ph - 1:ph - 1 + H, pw - 1:pw - 1 + W]


def _circ_adjoint(w, psf, dw, dh, N, M):
    ph, pw = psf.shape
    H, W = w.shape
    a = np.zeros((M, N))
    a[ph - 1:ph - 1 + H, pw - 1:pw - 1 + W] = w
    k = np.zeros((M, N))
    k[:ph, :pw] = psf
    c = np.real(np.fft.ifft2(np.fft.fft2(a) * np.conj(np.fft.fft2(k))))
    return c[:dh, :dw]


@pytest.mark.parametrize("W,H,pw,ph", [(20, 20, 7, 7), (17, 23, 6, 6), (12, 30, 9, 5), (25, 14, 4, 8)])
def test_drawing_sized_grid_reproduces_brute_force(W, H, pw, ph):
    r = np.random.Generator(np.random.PCG64(17))
    dw, dh = W + 2 * (pw // 2), H + 2 * (ph // 2)
    conv = r.normal(size=(dh, dw))
    psf = r.uniform(size=(ph, pw))
    w = r.normal(size=(H, W))
    # the smallest grid the argument allows: the drawing itself
    N, M = dw, dh
    fwd_b = _brute_forward(conv, psf, W, H)
    fwd_c = _circ_forward(conv, psf, W, H, N, M)
    np.testing.assert_allclose(fwd_c, fwd_b, rtol=0, atol=1e-12 * np.abs(fwd_b).max())
    adj_b = _brute_adjoint(w, psf, dw, dh)
    adj_c = _circ_adjoint(w, psf, dw, dh, N, M)
    np.testing.assert_allclose(adj_c, adj_b, rtol=0, atol=1e-12 * np.abs(adj_b).max())
    # a larger grid (as fft_good_size may give) changes nothing
    np.testing.assert_allclose(_circ_forward(conv, psf, W, H, N + 6, M + 4), fwd_b, rtol=0,
                               atol=1e-12 * np.abs(fwd_b).max())
    np.testing.assert_allclose(_circ_adjoint(w, psf, dw, dh, N + 6, M + 4), adj_b, rtol=0,
                               atol=1e-12 * np.abs(adj_b).max())

