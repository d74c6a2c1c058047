"""CPU oracle (test infrastructure only; never imported by the product path)
for the 3-D periodic particle-mesh force, the f64 Ewald direct sum that
judges it, and the per-particle MLP short-range correction.

The PM cycle follows the reference's plan for the mesh code (TODO.md:225-253:
CIC deposit, Poisson solve phi_k = -4 pi G rho_k / k^2 with the k = 0 term
set to zero, CIC interpolation with the deposit's stencil) and its 2-D
implementation (backend/pm_kernel.py:63-90 deposit, :93-107 gather,
:127-147 field), made periodic in 3-D: corners wrap instead of clipping,
the Green's function is divided by the CIC window twice (deposit and
interpolation; "Green's function must match the CIC discretisation",
TODO.md:243-246) and filtered by the long-range Gaussian exp(-k^2 r_s^2),
and the gradient is taken spectrally (a_d = -i k_d phi_k, zero on the
axis's own Nyquist plane). All arithmetic here is f64 NumPy.

The direct sum for a periodic box is the Ewald sum (Hernquist, Bouchet &
Suto 1991, ApJS 75:231): real-space erfc part over images inside r_cut,
reciprocal part over k = 2 pi h / L with |h| <= h_max, plus the Plummer
softening applied to the nearest image of every pair as
(r^2 + eps^2)^(-3/2) - r^-3 (so the result does not depend on alpha).

The P3M pair term (p3m_short) has no reference counterpart: it is the
exact complement of the Gaussian-filtered mesh force (the Ewald real-space
term with alpha = 1 / (2 r_s)) plus the softening, inside r_cut.

The MLP restatement (67 -> 128 -> 128 -> 3, SiLU) rounds to bf16 at exactly
the points where the tensor-core kernels do (inputs, weights, hidden
activations, output and hidden deltas), so its gradients are comparable with
the GPU's to f32 accumulation error.
"""
from __future__ import annotations

import itertools
import math

import numpy as np
from scipy.special import erf, erfc

# ------------------------------------------------------------- PM

CORNERS = list(itertools.product((0, 1), repeat=3))


def _cells(pos, n, L):
    f = np.asarray(pos, np.float64) * (n / L)
    i0 = np.floor(f)
    t = f - i0
    return i0.astype(np.int64) % n, t


def cic_deposit(pos, mass, n, L=1.0):
    """Density mesh (n, n, n) = sum of CIC-weighted masses / h^3, periodic."""
    i0, t = _cells(pos, n, L)
    rho = np.zeros(n ** 3)
    m = np.asarray(mass, np.float64)
    for dx, dy, dz in CORNERS:
        w = (np.where(dx, t[:, 0], 1.0 - t[:, 0]) * np.where(dy, t[:, 1], 1.0 - t[:, 1])
             * np.where(dz, t[:, 2], 1.0 - t[:, 2]))
        idx = (((i0[:, 0] + dx) % n) * n + (i0[:, 1] + dy) % n) * n + (i0[:, 2] + dz) % n
        rho += np.bincount(idx, weights=m * w, minlength=n ** 3)
    h = L / n
    return (rho / h ** 3).reshape(n, n, n)


def wavenumbers(n, L=1.0):
    """k_d of the full axes (numpy fftfreq order) and of the half axis."""
    kf = 2.0 * np.pi / L * np.fft.fftfreq(n, 1.0 / n)
    kh = 2.0 * np.pi / L * np.arange(n // 2 + 1)
    return kf, kh


def force_meshes(rho, G=1.0, L=1.0, deconv=2, r_split=0.0):
    """Acceleration meshes (3, n, n, n) from a periodic density mesh with the
    Green's function -4 pi G / k^2 * W(k)^-deconv * exp(-k^2 r_split^2)
    (W = the CIC window; the Gaussian is the long-range filter that keeps
    the deconvolution from amplifying the mesh-scale aliasing)."""
    n = rho.shape[0]
    h = L / n
    rk = np.fft.rfftn(rho)
    kf, kh = wavenumbers(n, L)
    kx = kf[:, None, None]
    ky = kf[None, :, None]
    kz = kh[None, None, :]
    k2 = kx ** 2 + ky ** 2 + kz ** 2
    green = np.zeros_like(k2)
    nz = k2 > 0
    green[nz] = -4.0 * np.pi * G / k2[nz]
    if deconv:
        def sinc(k):
            x = 0.5 * k * h
            return np.where(x == 0.0, 1.0, np.sin(x) / np.where(x == 0.0, 1.0, x))
        w = (sinc(kx) * sinc(ky) * sinc(kz)) ** 2
        green = green / w ** deconv
    if r_split > 0.0:
        green = green * np.exp(-k2 * r_split * r_split)
    phi = green * rk
    out = np.empty((3, n, n, n))
    nyq = n // 2
    for d, kd in enumerate((kx, ky, kz)):
        ad = -1j * kd * phi
        ad = ad.copy()
        if d == 0:
            ad[nyq, :, :] = 0.0
        elif d == 1:
            ad[:, nyq, :] = 0.0
        else:
            ad[:, :, nyq] = 0.0
        out[d] = np.fft.irfftn(ad, s=(n, n, n), axes=(0, 1, 2))
    return out


def cic_gather(meshes, pos, L=1.0):
    """Trilinear (CIC) interpolation of 3 meshes at pos -> (N, 3)."""
    n = meshes.shape[1]
    i0, t = _cells(pos, n, L)
    flat = meshes.reshape(3, -1)
    out = np.zeros((len(i0), 3))
    for dx, dy, dz in CORNERS:
        w = (np.where(dx, t[:, 0], 1.0 - t[:, 0]) * np.where(dy, t[:, 1], 1.0 - t[:, 1])
             * np.where(dz, t[:, 2], 1.0 - t[:, 2]))
        idx = (((i0[:, 0] + dx) % n) * n + (i0[:, 1] + dy) % n) * n + (i0[:, 2] + dz) % n
        out += w[:, None] * flat[:, idx].T
    return out


def pm_accel(pos, mass, n, G=1.0, L=1.0, deconv=2, r_split=None):
    """Mesh accelerations at the particles; r_split None = 0.6 cells."""
    rho = cic_deposit(pos, mass, n, L)
    rs = 0.6 * L / n if r_split is None else r_split
    return cic_gather(force_meshes(rho, G, L, deconv, rs), pos, L)


def wrap(x, L=1.0):
    return x - L * np.floor(x / L)


def kdk(pos, vel, acc, mass, dt, steps, n, G=1.0, L=1.0, accel=None, deconv=2, r_split=None):
    """KDK leapfrog with PM forces (as NBodyPM, pm_kernel.py:166-293, made
    periodic): v += a dt/2; x += v dt (wrapped); a = F(x); v += a dt/2."""
    x = np.array(pos, np.float64)
    v = np.array(vel, np.float64)
    a = np.array(acc, np.float64)
    accel = accel or (lambda p: pm_accel(p, mass, n, G, L, deconv, r_split))
    for _ in range(steps):
        v = v + a * (0.5 * dt)
        x = wrap(x + v * dt, L)
        a = accel(x)
        v = v + a * (0.5 * dt)
    return x, v, a


# ------------------------------------------------------------- Ewald


def ewald_hvectors(h_max):
    """Half-space integer vectors 0 < |h| <= h_max (one of each +-h pair)."""
    r = np.arange(-h_max, h_max + 1)
    hx, hy, hz = np.meshgrid(r, r, r, indexing="ij")
    h = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], 1)
    h2 = (h ** 2).sum(1)
    half = (h[:, 0] > 0) | ((h[:, 0] == 0) & (h[:, 1] > 0)) | ((h[:, 0] == 0) & (h[:, 1] == 0) & (h[:, 2] > 0))
    return h[half & (h2 <= h_max * h_max)]


def ewald_pair(r2, alpha, eps2, rc2, near_image=True):
    """The real-space factor f(r) of one source image, a = -G m f(r) d:
    the erfc part of the Ewald split, [erfc(x) + 2x/sqrt(pi) e^{-x^2}] / r^3
    (x = alpha r, r < r_cut), plus, on the nearest image, the Plummer
    correction (r^2 + eps^2)^{-3/2} - r^{-3} for every pair. Close pairs use
    the combined form (-erf(x) + 2x/sqrt(pi) e^{-x^2}) / r^3 +
    (r^2 + eps^2)^{-3/2}, which avoids the cancellation of the two 1/r^3."""
    r2 = np.asarray(r2, np.float64)
    r = np.sqrt(r2)
    x = alpha * r
    sp = 2.0 / math.sqrt(math.pi)
    inv_r3 = 1.0 / (r2 * r)
    gauss = sp * x * np.exp(-x * x)
    if not near_image:
        return np.where(r2 < rc2, (erfc(x) + gauss) * inv_r3, 0.0)
    small = r2 < max(1000.0 * eps2, (0.5 / alpha) ** 2)
    close = (-erf(x) + gauss) * inv_r3 + (r2 + eps2) ** -1.5
    soft = np.expm1(-1.5 * np.log1p(eps2 / r2)) * inv_r3
    far = soft + np.where(r2 < rc2, (erfc(x) + gauss) * inv_r3, 0.0)
    return np.where(small, close, far)


def p3m_short(src, mass, tgt, alpha, r_cut, G=1.0, L=1.0, eps=0.0, self_index=None):
    """The P3M pair term at tgt (T, 3), f64: over the sources closer than
    r_cut (nearest image, r_cut <= L / 3), a += G m (erfc(x) + 2x/sqrt(pi)
    e^{-x^2} + (1 + eps^2/r^2)^{-3/2} - 1) d / r^3 with x = alpha r and
    d = x_j - x_i; coincident pairs and self_index[i] are skipped. No
    reference counterpart: the exact complement of the mesh force filtered
    by exp(-k^2 r_split^2), r_split = 1 / (2 alpha) (the Ewald real-space
    term of ewald_pair with the softening kept inside r_cut)."""
    src = np.asarray(src, np.float64)
    tgt = np.asarray(tgt, np.float64)
    m = np.asarray(mass, np.float64)
    out = np.zeros((len(tgt), 3))
    eps2 = float(eps) ** 2
    sp = 2.0 / math.sqrt(math.pi)
    for i in range(len(tgt)):
        d = src - tgt[i]
        d = d - L * np.rint(d / L)
        r2 = (d * d).sum(1)
        keep = (r2 > 0.0) & (r2 < r_cut * r_cut)
        if self_index is not None and self_index[i] >= 0:
            keep[self_index[i]] = False
        r2k = r2[keep]
        r = np.sqrt(r2k)
        x = alpha * r
        g = erfc(x) + sp * x * np.exp(-x * x) + np.expm1(-1.5 * np.log1p(eps2 / r2k))
        out[i] = G * ((m[keep] * g / (r2k * r)) @ d[keep])
    return out


def ewald_accel(src, mass, tgt, G=1.0, L=1.0, alpha=10.0, r_cut=0.46, h_max=17, eps=0.0,
                images=0, self_index=None, chunk=2048):
    """Periodic accelerations at tgt (T, 3) from sources (N, 3), f64.

    images = 0: the erfc part on the nearest image only (needs r_cut <=
    L/2); images = 1: on the 27 boxes around the nearest image (r_cut <= L).
    The Plummer correction acts on the nearest image of every pair.
    self_index[i] = source index of target i (skipped) or -1."""
    src = np.asarray(src, np.float64)
    tgt = np.asarray(tgt, np.float64)
    m = np.asarray(mass, np.float64)
    T = len(tgt)
    out = np.zeros((T, 3))
    eps2 = float(eps) * float(eps)
    rc2 = float(r_cut) ** 2
    shifts = [(0, 0, 0)] if images == 0 else list(itertools.product((-1, 0, 1), repeat=3))
    for i in range(T):
        d0 = tgt[i] - src
        d0 = d0 - L * np.rint(d0 / L)          # nearest image; other boxes are shifts of it
        acc = np.zeros(3)
        for s in shifts:
            d = d0 + L * np.asarray(s, np.float64)
            r2 = (d * d).sum(1)
            keep = r2 > 0.0
            nearest = s == (0, 0, 0)
            if self_index is not None and self_index[i] >= 0 and nearest:
                keep[self_index[i]] = False
            if not nearest:
                keep &= r2 < rc2
            f = ewald_pair(r2[keep], alpha, eps2, rc2, nearest)
            acc -= G * (m[keep] * f) @ d[keep]
        out[i] = acc
    # reciprocal part
    h = ewald_hvectors(h_max).astype(np.float64)
    k = 2.0 * np.pi / L * h
    k2 = (k * k).sum(1)
    coef = 2.0 * 4.0 * np.pi / L ** 3 * np.exp(-k2 / (4.0 * alpha * alpha)) / k2
    for c0 in range(0, len(k), chunk):
        kc = k[c0:c0 + chunk]
        ph = src @ kc.T                       # (N, nk)
        C = m @ np.cos(ph)
        S = m @ np.sin(ph)
        pt = tgt @ kc.T                       # (T, nk)
        f = np.sin(pt) * C - np.cos(pt) * S   # sum_j m_j sin(k.(x_i - x_j))
        out -= G * (f * coef[c0:c0 + chunk]) @ kc
    return out


# ------------------------------------------------------------- MLP

N_IN = 67          # 4x4x4 density patch + 3 sub-cell offsets
K1 = 80            # padded input width (multiple of 16)
HID = 128
N_OUT = 3
K3 = 8             # padded output width
SHAPES = (("W1", (K1, HID)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (HID, K3)), ("b3", (K3,)))
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(params):
    p = np.asarray(params, np.float64)
    out, o = {}, 0
    for name, s in SHAPES:
        c = int(np.prod(s))
        out[name] = p[o:o + c].reshape(s)
        o += c
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def bf16(x):
    """Round to the nearest bf16 (ties to even), returned as f64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def features(pos, rho, rho_mean, L=1.0):
    """(N, 80) inputs: log1p(rho/rho_mean) on the 4x4x4 cells (i0-1 .. i0+2)
    around the particle's cell, then the sub-cell offsets - 1/2, then 0."""
    n = rho.shape[0]
    i0, t = _cells(pos, n, L)
    N = len(i0)
    X = np.zeros((N, K1))
    flat = np.log1p(rho.reshape(-1) / rho_mean)
    c = 0
    for a in range(4):
        for b in range(4):
            for e in range(4):
                idx = (((i0[:, 0] + a - 1) % n) * n + (i0[:, 1] + b - 1) % n) * n + (i0[:, 2] + e - 1) % n
                X[:, c] = flat[idx]
                c += 1
    X[:, 64:67] = t - 0.5
    return X


def forward(params, X, emulate=True):
    """Y (N, 3) and the cache for backward. emulate=False: exact f64."""
    q = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    p = unpack(params)
    W1, W2, W3 = q(p["W1"]), q(p["W2"]), q(p["W3"])
    X = q(X)
    Z1 = X @ W1 + p["b1"]
    H1 = q(silu(Z1))
    Z2 = H1 @ W2 + p["b2"]
    H2 = q(silu(Z2))
    Y = H2 @ W3 + p["b3"]
    return Y[:, :N_OUT], dict(X=X, Z1=Z1, H1=H1, Z2=Z2, H2=H2, W1=W1, W2=W2, W3=W3, Y=Y)


def loss(Y, T):
    return float(np.mean((Y - T) ** 2))


def backward(params, cache, T, emulate=True):
    """Gradient of mean((Y - T)^2) over samples and the 3 outputs, in the
    flat parameter layout."""
    q = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    N = len(T)
    dY = np.zeros((N, K3))
    dY[:, :N_OUT] = 2.0 * (cache["Y"][:, :N_OUT] - T) / (N * N_OUT)
    dY = q(dY)
    dH2 = dY @ cache["W3"].T
    dZ2 = q(dH2 * dsilu(cache["Z2"]))
    dH1 = dZ2 @ cache["W2"].T
    dZ1 = q(dH1 * dsilu(cache["Z1"]))
    g = dict(W1=cache["X"].T @ dZ1, b1=dZ1.sum(0), W2=cache["H1"].T @ dZ2, b2=dZ2.sum(0),
             W3=cache["H2"].T @ dY, b3=dY.sum(0))
    return pack(g)


def adam(params, grads, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba 2015), t counted from 1; returns copies."""
    m = b1 * m + (1 - b1) * grads
    v = b2 * v + (1 - b2) * grads * grads
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v


def init_params(seed=0):
    """He-style uniform init; padded rows/columns are zero and stay zero."""
    rng = np.random.default_rng(seed)
    d = {}
    w1 = np.zeros((K1, HID))
    w1[:N_IN] = rng.uniform(-1, 1, (N_IN, HID)) * math.sqrt(6.0 / N_IN)
    d["W1"] = w1
    d["b1"] = np.zeros(HID)
    d["W2"] = rng.uniform(-1, 1, (HID, HID)) * math.sqrt(6.0 / HID)
    d["b2"] = np.zeros(HID)
    w3 = np.zeros((HID, K3))
    w3[:, :N_OUT] = rng.uniform(-1, 1, (HID, N_OUT)) * math.sqrt(1.0 / HID)
    d["W3"] = w3
    d["b3"] = np.zeros(K3)
    return pack(d).astype(np.float32).astype(np.float64)


def median_rel_err(a, ref):
    """Median over particles of |a - ref| / |ref| (vector norms)."""
    return float(np.median(np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)))
