"""CPU oracle: a numpy restatement of QoraHolo's CPU path (hologram -> refractive index and the BPM
inversion), used only as the checker of the CUDA path.

TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module. The product (qoraholo_b200) never calls it and has no CPU fallback.

Every function names the reference function it follows (paths within the QoraHolo sources). Float
arithmetic is float32 in the same order as the C++ where that order decides rounding: the Ewald
indices (src/common.hpp:56-67), the accumulation order of the mapping (src/cpu/odt.cpp:147-161),
the FGP dual step (src/common.hpp:107-153, src/cpu/tv.cpp:7-44). FFTs are scipy.fft, which is the
pocketfft family the reference links (pinned pocketfft commit 4d865cba, CMakeLists.txt:27-33), in
single precision; transcendental functions are evaluated in float64 and rounded once, which is
what a correctly rounded libm returns. The restatement is pinned against the reference itself:
tests/test_oracle.py compares it with oracle/_ref (the reference sources compiled here) and with
the golden fixtures in tests/golden/ that oracle/_ref produced.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.fft as sfft

F32 = np.float32
C64 = np.complex64
PI_F = F32(3.14159265358979323846)  # kPi, src/common.hpp:16
TWO_PI_F = F32(2.0) * PI_F
WORKERS = -1  # scipy.fft threads: all cores, as pocketfft's threads() (src/cpu/fft.cpp:10-13)


def _f(x):
    return F32(x)


# ---------------------------------------------------------------------------------------------
# shared math, src/common.hpp


def parity(i):
    """(-1)^i, src/common.hpp:19."""
    return np.where(np.asarray(i) & 1, F32(-1.0), F32(1.0)).astype(F32)


def signed_bin(k, n):
    """src/common.hpp:22."""
    k = np.asarray(k)
    return np.where(k < n // 2, k, k - n)


def dct_position(i, n):
    """Makhoul reordering, src/common.hpp:25."""
    i = np.asarray(i)
    return np.where(i & 1, n - 1 - (i >> 1), i >> 1)


def _cosf(x):
    return np.cos(np.asarray(x, np.float64)).astype(F32)


def _sinf(x):
    return np.sin(np.asarray(x, np.float64)).astype(F32)


def neumann_eigenvalue(ky, kx, ny, nx):
    """src/common.hpp:28-31."""
    a = F32(2.0) * _cosf(PI_F * np.asarray(ky, F32) / F32(ny))
    b = F32(2.0) * _cosf(PI_F * np.asarray(kx, F32) / F32(nx))
    return (a + b - F32(4.0)).astype(F32)


def wrap_phase(p):
    """src/common.hpp:33."""
    p = np.asarray(p, F32)
    return (p - TWO_PI_F * np.floor((p + PI_F) / TWO_PI_F).astype(F32)).astype(F32)


def make_grid(n, nz, geom):
    """src/api.cpp:32-42: (n, nz, df, dfz, fm2, fna2, gain) in float."""
    wavelength, n_medium, na, pixel = (F32(v) for v in geom)
    fm = n_medium / wavelength
    fna = na / wavelength
    return dict(n=n, nz=nz, df=F32(1.0) / (F32(n) * pixel), dfz=F32(1.0) / (F32(nz) * pixel),
                fm2=fm * fm, fna2=fna * fna, gain=F32(4.0) * F32(math.pi) / pixel)


def ewald_targets(g, fiy, fix, fiz):
    """ewald_target (src/common.hpp:56-67) for every lateral bin (ky, kx) of one illumination.
    Returns (valid mask, kz wrapped to [0, nz), nu_z), each (n, n)."""
    n, nz = g["n"], g["nz"]
    sb = signed_bin(np.arange(n), n).astype(F32)
    fy = (sb * g["df"] + F32(fiy))[:, None]
    fx = (sb * g["df"] + F32(fix))[None, :]
    rho2 = (fy * fy + fx * fx).astype(F32)
    ok = ~((rho2 > g["fna2"]) | (rho2 >= g["fm2"]))
    nuz = np.sqrt(np.where(ok, g["fm2"] - rho2, F32(0.0))).astype(F32)
    k = np.floor((nuz - F32(fiz)) / g["dfz"] + F32(0.5)).astype(np.int64)
    ok &= (k >= -(nz // 2)) & (k < nz // 2)
    kz = np.where(k < 0, k + nz, k)
    return ok, kz, nuz


def hermitian_data(pre, pim, nre, nim):
    """src/common.hpp:79-82."""
    return F32(0.5) * (pre + nre), F32(0.5) * (pim - nim)


def hermitian_restore(are, aim, hits, re, im):
    """src/common.hpp:83-87."""
    b = F32(1.0) - F32(0.5) * hits.astype(F32)
    return are + b * re, aim + b * im


def fista_t(t):
    """src/common.hpp:153."""
    t = F32(t)
    return F32(0.5) * (F32(1.0) + np.sqrt(F32(1.0) + F32(4.0) * t * t))


def index_from_potential(re, im, nm2, inv_k02):
    """src/common.hpp:179-183."""
    a = F32(nm2) + np.asarray(re, F32) * F32(inv_k02)
    b = np.asarray(im, F32) * F32(inv_k02)
    h = np.hypot(a.astype(np.float64), b.astype(np.float64)).astype(F32)
    return np.sqrt(F32(0.5) * (h + a)).astype(F32)


# ---------------------------------------------------------------------------------------------
# FFT helpers with the reference's conventions, src/cpu/fft.cpp


def fft(a, axes, forward=True, scale=1.0):
    """cpu::fft (src/cpu/fft.cpp:18-28): unnormalised c2c over `axes`, times scale."""
    a = np.asarray(a, C64)
    out = sfft.fftn(a, axes=axes, workers=WORKERS) if forward else sfft.ifftn(a, axes=axes, norm="forward", workers=WORKERS)
    out = out.astype(C64, copy=False)
    if scale != 1.0:
        out = (out * F32(scale)).astype(C64)
    return out


def rfft3(x):
    """cpu::rfft3 (src/cpu/fft.cpp:49-54): real (nz, ny, nx) -> half spectrum (nz, ny, nx/2+1)."""
    return sfft.rfftn(np.asarray(x, F32), axes=(0, 1, 2), workers=WORKERS).astype(C64, copy=False)


def irfft3(e, shape, scale):
    """cpu::irfft3 (src/cpu/fft.cpp:56-66): half spectrum -> real, times scale."""
    y = sfft.ifftn(np.asarray(e, C64), axes=(0, 1), norm="forward", workers=WORKERS)
    x = sfft.irfft(y, n=shape[2], axis=2, norm="forward", workers=WORKERS).astype(F32, copy=False)
    return (x * F32(scale)).astype(F32)


def _dct_twiddles(n, sign):
    k = np.arange(n, dtype=np.float64)
    a = sign * math.pi * k / (2.0 * n)
    return (np.cos(a).astype(F32) + 1j * np.sin(a).astype(F32)).astype(C64)


def dct2(a, axis):
    """Makhoul DCT-II via FFT along axis 1 (y) or 2 (x), src/cpu/fft.cpp:101-115."""
    a = np.asarray(a, F32)
    n = a.shape[axis]
    pos = dct_position(np.arange(n), n)
    buf = np.zeros(a.shape, C64)
    idx = [slice(None)] * 3
    idx[axis] = pos
    buf[tuple(idx)] = a
    buf = fft(buf, (axis,), True)
    w = _dct_twiddles(n, -1.0)
    shape = [1, 1, 1]
    shape[axis] = n
    w = w.reshape(shape)
    return (w.real * buf.real - w.imag * buf.imag).astype(F32)


def idct2(a, axis):
    """Inverse of dct2, src/cpu/fft.cpp:117-133."""
    a = np.asarray(a, F32)
    n = a.shape[axis]
    mirror = np.flip(a, axis=axis)  # a[n - 1 - k]
    mirror = np.roll(mirror, 1, axis=axis)  # a[n - k] at k, a[0] at k = 0
    idx = [slice(None)] * 3
    idx[axis] = 0
    mirror[tuple(idx)] = 0.0
    v = (a + 1j * (-mirror)).astype(C64)
    w = _dct_twiddles(n, 1.0)
    shape = [1, 1, 1]
    shape[axis] = n
    buf = (w.reshape(shape) * v).astype(C64)
    buf = fft(buf, (axis,), False, F32(1.0) / F32(n))
    pos = dct_position(np.arange(n), n)
    idx[axis] = pos
    return buf[tuple(idx)].real.astype(F32)


# ---------------------------------------------------------------------------------------------
# field retrieval, src/api.cpp:52-81 and src/cpu/field.cpp


def crop_plan(center, n, radius=0.0, output_size=0):
    """src/api.cpp:52-60: (cy, cx, radius, out)."""

    def lround(v):
        return int(math.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)

    cy, cx = lround(float(F32(center[0]))), lround(float(F32(center[1])))
    out = output_size if output_size > 0 else n
    r = F32(radius)
    if r <= 0:
        r = F32(np.hypot(np.float64(F32(center[0])), np.float64(F32(center[1])))) / F32(3.0)
    if not (out % 2 == 0 and out <= n):
        raise ValueError("extract_fields: output_size must be even and <= N")
    if not (r > 0 and r <= F32(out) / F32(2.0)):
        raise ValueError("extract_fields: crop radius must fit in the output window")
    return cy, cx, F32(r), out


def _shifted_spectra(h):
    n = h.shape[-1]
    y, x = np.indices((n, n))
    s = (np.asarray(h, F32) * parity(x + y)).astype(C64)
    return fft(s, (-2, -1), True)


def _refine(lo, mid, hi, n):
    """Jacobsen / Candan, src/cpu/field.cpp:15-22."""
    den = C64(2.0) * C64(mid) - C64(lo) - C64(hi)
    if abs(den) == 0.0:
        return F32(0.0)
    c = PI_F / F32(n)
    d = F32(((C64(lo) - C64(hi)) / den).real) * F32(math.tan(float(c))) / c
    return F32(min(max(d, -0.5), 0.5))


def find_sideband(holograms, dc_exclusion=0.0):
    """src/cpu/field.cpp:25-60. Returns (iy, ix, y, x, magnitude)."""
    h = np.asarray(holograms, F32)
    if h.ndim == 2:
        h = h[None]
    n = h.shape[2]
    if h.shape[0] < 1 or h.shape[1] != n or n % 2 or n < 4:
        raise ValueError("find_sideband: holograms must be square with an even side")
    dc = F32(dc_exclusion) if dc_exclusion > 0 else F32(n) / F32(8.0)
    s = _shifted_spectra(h[0])
    c = n // 2
    mag = np.abs(s.astype(np.complex128)).astype(F32)
    best = (0, 0, F32(0.0))
    for y in range(1, n - 1):
        for x in range(c, n - 1):
            dy, dx = y - c, x - c
            if dx == 0 and dy <= 0:
                continue
            if F32(dy * dy + dx * dx) <= dc * dc:
                continue
            if mag[y, x] > best[2]:
                best = (dy, dx, mag[y, x])
    if best[2] == 0:
        raise RuntimeError("find_sideband: no peak outside the DC region")
    iy, ix, m = best
    y, x = iy + c, ix + c
    fy = F32(iy) + _refine(s[y - 1, x], s[y, x], s[y + 1, x], n)
    fx = F32(ix) + _refine(s[y, x - 1], s[y, x], s[y, x + 1], n)
    return iy, ix, float(fy), float(fx), float(m)


def extract_fields(holograms, center=None, radius=0.0, dc_exclusion=0.0, output_size=0):
    """extract_fields (src/api.cpp:62-81) -> cpu::extract_fields (src/cpu/field.cpp:78-121)."""
    h = np.asarray(holograms, F32)
    if h.ndim == 2:
        h = h[None]
    nz, ny, n = h.shape
    if not (ny == n and n >= 4 and n % 2 == 0):
        raise ValueError("extract_fields: images must be square with an even side")
    if center is None:
        iy, ix, *_ = find_sideband(h, dc_exclusion)
        center = (float(iy), float(ix))
    cy, cx, r, m = crop_plan(center, n, radius, output_size)
    spec = _shifted_spectra(h)
    sign = parity(cy + cx)
    r2 = r * r
    dy = (np.arange(m) - m // 2)[:, None]
    dx = (np.arange(m) - m // 2)[None, :]
    sy = n // 2 + cy + dy
    sx = n // 2 + cx + dx
    inside = ((dy * dy + dx * dx).astype(F32) <= r2) & (sy >= 0) & (sy < n) & (sx >= 0) & (sx < n)
    out = np.zeros((nz, m, m), C64)
    yy, xx = np.nonzero(inside)
    out[:, yy, xx] = spec[:, sy[yy, 0], sx[0, xx]] * sign
    out = fft(out, (1, 2), False, F32(1.0) / F32(n * n))
    y, x = np.indices((m, m))
    return (out * parity(x + y)).astype(C64)


def field_ratio(sample, background):
    """src/cpu/field.cpp:62-74."""
    s = np.asarray(sample, C64)
    b = np.asarray(background, C64)
    if s.ndim == 2:
        s = s[None]
    if b.ndim == 2:
        b = b[None]
    if s.shape[1:] != b.shape[1:] or (b.shape[0] != 1 and b.shape[0] != s.shape[0]):
        raise ValueError("field_ratio: background shape does not match")
    return (s / b).astype(C64)


# ---------------------------------------------------------------------------------------------
# unwrapping and Rytov, src/cpu/unwrap.cpp


def unwrap(psi):
    """src/cpu/unwrap.cpp:11-59: least-squares (DCT) unwrap + congruence constant."""
    psi = np.asarray(psi, F32)
    if psi.ndim == 2:
        psi = psi[None]
    nz, ny, nx = psi.shape
    if ny % 2 or nx % 2 or ny < 2 or nx < 2:
        raise ValueError("unwrap: image sides must be even")
    r = np.zeros_like(psi)
    r[:, :, :-1] += wrap_phase(psi[:, :, 1:] - psi[:, :, :-1])
    r[:, :, 1:] -= wrap_phase(psi[:, :, 1:] - psi[:, :, :-1])
    r[:, :-1, :] += wrap_phase(psi[:, 1:, :] - psi[:, :-1, :])
    r[:, 1:, :] -= wrap_phase(psi[:, 1:, :] - psi[:, :-1, :])
    phi = dct2(r, 2)
    phi = dct2(phi, 1)
    ky = np.arange(ny)[:, None]
    kx = np.arange(nx)[None, :]
    ev = neumann_eigenvalue(ky, kx, ny, nx)
    ev[0, 0] = 1.0
    phi = (phi / ev).astype(F32)
    phi[:, 0, 0] = 0.0
    phi = idct2(phi, 1)
    phi = idct2(phi, 2)
    d = (psi - phi).astype(F32).astype(np.float64).reshape(nz, -1)
    acc = np.exp(1j * d).sum(axis=1)
    c = np.angle(acc).astype(F32)
    return (phi + c[:, None, None]).astype(F32)


def rytov(ratio):
    """src/cpu/unwrap.cpp:61-82: log|r| + i (unwrap(arg r) - 2 pi m), m from the border mean."""
    r = np.asarray(ratio, C64)
    if r.ndim == 2:
        r = r[None]
    nz, ny, nx = r.shape
    if ny % 2 or nx % 2 or ny < 4 or nx < 4:
        raise ValueError("rytov: image sides must be even")
    r64 = r.astype(np.complex128)
    wrapped = np.arctan2(r64.imag, r64.real).astype(F32)
    phase = unwrap(wrapped)
    border = (phase[:, 0, :].astype(np.float64).sum(1) + phase[:, ny - 1, :].astype(np.float64).sum(1)
              + phase[:, 1:ny - 1, 0].astype(np.float64).sum(1) + phase[:, 1:ny - 1, nx - 1].astype(np.float64).sum(1))
    mean = border / (2.0 * nx + 2.0 * (ny - 2))
    shift = (2.0 * math.pi * np.round(mean / (2.0 * math.pi))).astype(F32)
    logamp = np.log(np.abs(r).astype(F32).astype(np.float64)).astype(F32)
    return (logamp + 1j * (phase - shift[:, None, None])).astype(C64)


# ---------------------------------------------------------------------------------------------
# ODT, src/api.cpp:107-137 and src/cpu/odt.cpp


def odt_grid(n, count, illuminations, geom, nz=0):
    """Validation of src/api.cpp:107-123."""
    if not (n >= 4 and n % 2 == 0):
        raise ValueError("reconstruct: images must be square with an even side")
    il = np.asarray(illuminations, F32).reshape(-1, 2)
    if not (count >= 1 and il.shape[0] == count):
        raise ValueError("reconstruct: need one illumination per field")
    wavelength, n_medium, na, pixel = geom
    if not (wavelength > 0 and pixel > 0 and n_medium > 0 and na > 0):
        raise ValueError("reconstruct: geometry values must be positive")
    nzz = nz if nz > 0 else n
    if nzz % 2:
        raise ValueError("reconstruct: nz must be even")
    fm = F32(n_medium) / F32(wavelength)
    for fy, fx in il:
        if not (fy * fy + fx * fx < fm * fm):
            raise ValueError("reconstruct: illumination frequency beyond n_medium / wavelength")
    return make_grid(n, nzz, geom)


def illumination_fiz(g, illuminations):
    """fiz of each illumination in float (src/cpu/odt.cpp:141-144)."""
    il = np.asarray(illuminations, F32).reshape(-1, 2)
    return np.sqrt(g["fm2"] - il[:, 0] * il[:, 0] - il[:, 1] * il[:, 1]).astype(F32)


def ewald_map(spectra, illuminations, g):
    """Column-owner mapping (src/cpu/odt.cpp:147-161): full complex potential (nz, n, n) summed in
    illumination order, and the hit counts."""
    n, nz = g["n"], g["nz"]
    il = np.asarray(illuminations, F32).reshape(-1, 2)
    fiz = illumination_fiz(g, il)
    pre = np.zeros((nz, n, n), F32)
    pim = np.zeros((nz, n, n), F32)
    weight = np.zeros((nz, n, n), F32)
    yy, xx = np.indices((n, n))
    for a in range(il.shape[0]):
        ok, kz, nuz = ewald_targets(g, il[a, 0], il[a, 1], fiz[a])
        f = -g["gain"] * nuz  # the imaginary factor (0, f) of src/cpu/odt.cpp:156
        s = spectra[a]
        vr = -(f * s.imag.astype(F32))
        vi = f * s.real.astype(F32)
        p = parity(kz)
        sel = np.nonzero(ok)
        k = kz[sel]
        pre[k, yy[sel], xx[sel]] += (p * vr)[sel]
        pim[k, yy[sel], xx[sel]] += (p * vi)[sel]
        weight[k, yy[sel], xx[sel]] += F32(1.0)
    return pre, pim, weight


def hermitian_half(pre, pim, weight):
    """hermitian_data (src/cpu/odt.cpp:37-62): half-spectrum data a and hits = M(k) + M(-k)."""
    nz, n, _ = pre.shape
    h = n // 2 + 1
    mz = (-np.arange(nz)) % nz
    my = (-np.arange(n)) % n
    mx = (-np.arange(h)) % n
    nre = pre[mz][:, my][:, :, mx]
    nim = pim[mz][:, my][:, :, mx]
    are, aim = hermitian_data(pre[:, :, :h], pim[:, :, :h], nre, nim)
    hits = (weight[:, :, :h] > 0).astype(np.uint8) + (weight[mz][:, my][:, :, mx] > 0).astype(np.uint8)
    return (are + 1j * aim).astype(C64), hits.astype(np.uint8)


def restore(e, a, hits):
    re, im = hermitian_restore(a.real, a.imag, hits, e.real, e.imag)
    return (re + 1j * im).astype(C64)


def gp_real(a, hits, nz, n, iterations):
    """src/cpu/odt.cpp:76-90."""
    inv = F32(1.0) / (F32(nz) * F32(n) * F32(n))
    x = irfft3(a, (nz, n, n), inv)
    for _ in range(iterations):
        x = np.maximum(x, F32(0.0))
        e = restore(rfft3(x), a, hits)
        x = irfft3(e, (nz, n, n), inv)
    return x


def tv_adjoint(qz, qy, qx):
    """L(q) = -div q (src/common.hpp:107-118), accumulated in the same order."""
    s = np.zeros_like(qz)
    s[:-1] += qz[:-1]
    s[1:] -= qz[:-1]
    s[:, :-1] += qy[:, :-1]
    s[:, 1:] -= qy[:, :-1]
    s[:, :, :-1] += qx[:, :, :-1]
    s[:, :, 1:] -= qx[:, :, :-1]
    return s


def tv_primal(b, lam, adj):
    """src/common.hpp:121-124."""
    x = (b - F32(lam) * adj).astype(F32)
    return np.where(x > F32(0.0), x, F32(0.0)).astype(F32)


def tv_gradient(x):
    """src/common.hpp:144-150."""
    g0 = np.zeros_like(x)
    g1 = np.zeros_like(x)
    g2 = np.zeros_like(x)
    g0[:-1] = x[:-1] - x[1:]
    g1[:, :-1] = x[:, :-1] - x[:, 1:]
    g2[:, :, :-1] = x[:, :, :-1] - x[:, :, 1:]
    return g0, g1, g2


def tv_dual_step(g, step, momentum, p, r):
    """src/common.hpp:128-141, in place on the lists p and r of three volumes."""
    step, momentum = F32(step), F32(momentum)
    q = [(r[a] + step * g[a]).astype(F32) for a in range(3)]
    norm2 = (F32(0.0) + q[0] * q[0]).astype(F32)
    norm2 = (norm2 + q[1] * q[1]).astype(F32)
    norm2 = (norm2 + q[2] * q[2]).astype(F32)
    big = norm2 > F32(1.0)
    scale = np.where(big, F32(1.0) / np.sqrt(np.where(big, norm2, F32(1.0))), F32(1.0)).astype(F32)
    for a in range(3):
        nxt = (q[a] * scale).astype(F32)
        r[a] = (nxt + momentum * (nxt - p[a])).astype(F32)
        p[a] = nxt


def tv_prox(b, p, lam, inner):
    """cpu::tv_prox (src/cpu/tv.cpp:7-44): FGP with warm start; p (list of three volumes) is
    updated in place. Returns x = argmin 0.5|x - b|^2 + lam TV(x), x >= 0."""
    lam = F32(lam)
    step = F32(1.0) / (F32(12.0) * lam)
    r = [c.copy() for c in p]
    t = F32(1.0)
    for _ in range(inner):
        x = tv_primal(b, lam, tv_adjoint(*r))
        t_next = fista_t(t)
        m = (t - F32(1.0)) / t_next
        tv_dual_step(tv_gradient(x), step, m, p, r)
        t = t_next
    return tv_primal(b, lam, tv_adjoint(*p))


def tv_real(a, hits, nz, n, iterations, lam, inner):
    """FISTA-TV on half spectra, src/cpu/odt.cpp:94-120."""
    inv = F32(1.0) / (F32(nz) * F32(n) * F32(n))
    y = irfft3(a, (nz, n, n), inv)
    x_prev = y.copy()
    p = [np.zeros_like(y) for _ in range(3)]
    t = F32(1.0)
    for _ in range(iterations):
        e = restore(rfft3(y), a, hits)
        y = irfft3(e, (nz, n, n), inv)
        x = tv_prox(y, p, lam, inner)
        t_next = fista_t(t)
        m = (t - F32(1.0)) / t_next
        y = (x + m * (x - x_prev)).astype(F32)
        x_prev = x
        t = t_next
    return x_prev


def reconstruct(fields, illuminations, geom, nz=0, iterations=0, solver="gp", gp_transform="r2c",
                tv_weight=1e-2, tv_inner=10):
    """reconstruct (src/api.cpp:125-137) -> cpu::reconstruct (src/cpu/odt.cpp:124-242).
    Returns (ri, filled)."""
    f = np.asarray(fields, C64)
    if f.ndim == 2:
        f = f[None]
    count, ny, n = f.shape
    if ny != n:
        raise ValueError("reconstruct: images must be square")
    g = odt_grid(n, count, illuminations, geom, nz)
    nz = g["nz"]
    spectra = fft(f, (1, 2), True)
    pre, pim, weight = ewald_map(spectra, illuminations, g)
    filled_mask = weight > 0
    pre = np.where(filled_mask, pre / np.where(filled_mask, weight, F32(1.0)), pre).astype(F32)
    pim = np.where(filled_mask, pim / np.where(filled_mask, weight, F32(1.0)), pim).astype(F32)
    filled = float(np.count_nonzero(filled_mask)) / float(pre.size)
    wavelength, n_medium = F32(geom[0]), F32(geom[1])
    k0 = F32(2.0) * F32(math.pi) / wavelength
    nm2 = n_medium * n_medium
    inv_k02 = F32(1.0) / (k0 * k0)
    tv = solver == "tv"
    if iterations > 0 and (tv or gp_transform == "r2c"):
        a, hits = hermitian_half(pre, pim, weight)
        if tv:
            x = tv_real(a, hits, nz, n, iterations, F32(tv_weight) * k0 * k0, tv_inner)
        else:
            x = gp_real(a, hits, nz, n, iterations)
        return index_from_potential(x, F32(0.0), nm2, inv_k02), filled
    pot = (pre + 1j * pim).astype(C64)
    inv = F32(1.0) / F32(pot.size)
    if iterations > 0:
        measured = pot.copy()
        pot = fft(pot, (0, 1, 2), False, inv)
        for _ in range(iterations):
            pot = np.maximum(pot.real, F32(0.0)).astype(C64)
            pot = fft(pot, (0, 1, 2), True)
            pot = np.where(filled_mask, measured, pot).astype(C64)
            pot = fft(pot, (0, 1, 2), False, inv)
    else:
        pot = fft(pot, (0, 1, 2), False, inv)
    return index_from_potential(pot.real, pot.imag, nm2, inv_k02), filled


def circular_scan(count, na_illumination, geom):
    """src/api.cpp:203-216."""
    wavelength, n_medium = geom[0], geom[1]
    if count < 1:
        raise ValueError("circular_scan: count must be positive")
    if not (0 <= na_illumination < n_medium):
        raise ValueError("circular_scan: na_illumination must be below n_medium")
    out = np.zeros((count, 2), F32)
    f = F32(na_illumination) / F32(wavelength)
    for i in range(1, count):
        phi = F32(2.0) * F32(math.pi) * F32(i - 1) / F32(count - 1)
        out[i] = (f * _sinf(phi), f * _cosf(phi))
    return out


# ---------------------------------------------------------------------------------------------
# BPM, src/bpm.cpp and src/cpu/bpm.cpp


def bpm_tables(n, nz, illuminations, geom, obliquity=True):
    """src/bpm.cpp:10-60, in double, cast to float."""
    il = np.asarray(illuminations, F32).reshape(-1, 2).astype(np.float64)
    lam = float(F32(geom[0]))
    fm = float(F32(geom[1])) / lam
    fna = float(F32(geom[2])) / lam
    d = float(F32(geom[3]))
    df = 1.0 / (n * d)
    nuz_min = math.sqrt(max(fm * fm - fna * fna, 0.01 * fm * fm))
    back = -(nz - 1 - nz // 2) * d
    count = il.shape[0]
    sb = signed_bin(np.arange(n), n).astype(np.float64)
    step = np.zeros((count, n, n), C64)
    last = np.zeros((count, n, n), C64)
    q = np.ones((count, n, n), F32)
    q0 = 0.0
    for a in range(count):
        fiy, fix = il[a]
        fiz = math.sqrt(fm * fm - fiy * fiy - fix * fix)
        fy = (sb * df + fiy)[:, None]
        fx = (sb * df + fix)[None, :]
        rho2 = fy * fy + fx * fx
        inside = rho2 < fm * fm
        nuz = np.sqrt(np.where(inside, fm * fm - rho2, 0.0))
        ph = 2.0 * math.pi * (nuz - fiz)
        step[a] = np.where(inside, np.exp(1j * ph * d), 0.0).astype(C64)
        last[a] = np.where(inside & (rho2 <= fna * fna), np.exp(1j * ph * back), 0.0).astype(C64)
        if obliquity:
            q[a] = np.where(inside, fm / np.maximum(nuz, nuz_min), 1.0).astype(F32)
        q0 += float(q[a, 0, 0]) * float(q[a, 0, 0])
    phase = F32(2.0 * math.pi / lam * d)
    lipschitz = F32(nz * float(phase) * float(phase) * q0 / count)
    return dict(n=n, nz=nz, count=count, phase=phase, step=step, last=last, q=q, lipschitz=lipschitz)


def _screens(x, phase):
    th = (F32(phase) * np.asarray(x, F32)).astype(np.float64)
    return (np.cos(th).astype(F32) + 1j * np.sin(th).astype(F32)).astype(C64)


def _bpm_step(c, q, a, s):
    """src/common.hpp:158-163 on whole planes."""
    tre = q * a.real + (F32(1.0) - q) * s.real
    tim = q * a.imag + (F32(1.0) - q) * s.imag
    return (c.real * tre - c.imag * tim + 1j * (c.real * tim + c.imag * tre)).astype(C64)


def _fft2(a, forward, scale=1.0):
    return fft(a, (-2, -1), forward, scale)


def _forward(t, screen, angles, store=False):
    """forward_angle (src/cpu/bpm.cpp:41-62) for a batch of illuminations at once."""
    n, nz = t["n"], t["nz"]
    plane = n * n
    inv = F32(1.0) / F32(plane)
    nb = len(angles)
    s = np.zeros((nb, n, n), C64)
    s[:, 0, 0] = plane
    w = np.ones((nb, n, n), C64)
    stored = np.zeros((nz, nb, n, n), C64) if store else None
    for k in range(nz):
        if k > 0:
            w = _fft2(s, False, inv)
        if store:
            stored[k] = w
        v = _fft2((screen[k] * w).astype(C64), True)
        c = (t["last"] if k == nz - 1 else t["step"])[angles]
        s = _bpm_step(c, t["q"][angles], v, s)
    return _fft2(s, False, inv), stored


def _adjoint(t, screen, angles, stored, r):
    """adjoint_angle (src/cpu/bpm.cpp:65-98); returns the gradient contribution summed over the
    batch of illuminations."""
    n, nz = t["n"], t["nz"]
    inv = F32(1.0) / F32(n * n)
    g = _fft2(r, True)
    back = np.zeros_like(g)
    grad = np.zeros((nz, n, n), F32)
    q = t["q"][angles]
    for k in range(nz - 1, -1, -1):
        c = (t["last"] if k == nz - 1 else t["step"])[angles]
        gi = (g + back) if k < nz - 1 else g
        ure = c.real * gi.real + c.imag * gi.imag
        uim = c.real * gi.imag - c.imag * gi.real
        b = (q * ure + 1j * (q * uim)).astype(C64)
        g = ((F32(1.0) - q) * ure + 1j * ((F32(1.0) - q) * uim)).astype(C64)
        b = _fft2(b, False, inv)
        v = (screen[k] * stored[k]).astype(C64)
        grad[k] = (t["phase"] * (v.real * b.imag - v.imag * b.real)).sum(axis=0)
        back = _fft2((np.conj(screen[k]) * b).astype(C64), True)
    return grad


def bpm_forward_contrast(x, t):
    """cpu::bpm_forward (src/cpu/bpm.cpp:133-139) on the contrast x = n - n_medium."""
    y, _ = _forward(t, _screens(x, t["phase"]), np.arange(t["count"]))
    return y


def bpm_forward(ri, illuminations, geom, obliquity=True):
    """bpm_forward (src/api.cpp:167-178)."""
    ri = np.asarray(ri, F32)
    nz, n = ri.shape[0], ri.shape[2]
    t = bpm_tables(n, nz, illuminations, geom, obliquity)
    return bpm_forward_contrast((ri - F32(geom[1])).astype(F32), t)


def bpm_vjp(x, r, t):
    """cpu::bpm_vjp (src/cpu/bpm.cpp:178-189): J^T r for the contrast x."""
    screen = _screens(x, t["phase"])
    angles = np.arange(t["count"])
    _, stored = _forward(t, screen, angles, store=True)
    return _adjoint(t, screen, angles, stored, np.asarray(r, C64))


def bpm_gradient(t, x, fields, first, last):
    """gradient (src/cpu/bpm.cpp:102-129): (grad, loss)."""
    screen = _screens(x, t["phase"])
    angles = np.arange(first, last)
    y, stored = _forward(t, screen, angles, store=True)
    y = (y - fields[first:last]).astype(C64)
    loss = float(np.sum(np.abs(y.astype(np.complex128)) ** 2))
    grad = _adjoint(t, screen, angles, stored, y)
    return (grad * (F32(1.0) / F32(last - first))).astype(F32), 0.5 * loss / t["count"]


def bpm_reconstruct(fields, illuminations, geom, initial, iterations=20, batch=0, step=1.0, tv_weight=0.0,
                    tv_inner=10, obliquity=True):
    """bpm_reconstruct (src/api.cpp:180-201) -> cpu::bpm_reconstruct (src/cpu/bpm.cpp:191-243).
    Returns (ri, loss)."""
    f = np.asarray(fields, C64)
    init = np.asarray(initial, F32)
    nz, n = init.shape[0], init.shape[2]
    t = bpm_tables(n, nz, illuminations, geom, obliquity)
    count = t["count"]
    batch = count if batch <= 0 or batch >= count else batch
    alpha = F32(step) / t["lipschitz"]
    tv = tv_weight > 0
    x = np.maximum((init - F32(geom[1])).astype(F32), F32(0.0))
    p = [np.zeros_like(x) for _ in range(3)]

    def prox(point, grad):
        z = (point - alpha * grad).astype(F32)
        return tv_prox(z, p, alpha * F32(tv_weight), tv_inner) if tv else np.maximum(z, F32(0.0))

    losses = []
    if batch == count:
        y = x.copy()
        tk = F32(1.0)
        for _ in range(iterations):
            grad, loss = bpm_gradient(t, y, f, 0, count)
            losses.append(loss)
            nxt = prox(y, grad)
            tn = fista_t(tk)
            m = (tk - F32(1.0)) / tn
            y = (nxt + m * (nxt - x)).astype(F32)
            x = nxt
            tk = tn
    else:
        for _ in range(iterations):
            total = 0.0
            for first in range(0, count, batch):
                grad, loss = bpm_gradient(t, x, f, first, min(first + batch, count))
                total += loss
                x = prox(x, grad)
            losses.append(total)
    return (x + F32(geom[1])).astype(F32), np.asarray(losses)


# ---------------------------------------------------------------------------------------------
# phantom and synthesiser (fixture generators), src/phantom.cpp


def _index_at(spheres, count, n_medium, z, y, x):
    n = np.full(np.broadcast(z, y, x).shape, float(n_medium))
    for s in spheres[:count]:
        dz, dy, dx = z - float(s[0]), y - float(s[1]), x - float(s[2])
        inside = dz * dz + dy * dy + dx * dx <= float(s[3]) * float(s[3])
        n = np.where(inside, float(s[4]), n)
    return n


def render_phantom(spheres, geom, nz, n):
    """src/phantom.cpp:84-100. spheres: rows of (z, y, x, radius, n)."""
    s = np.asarray(spheres, F32).reshape(-1, 5)
    d = float(F32(geom[3]))
    k, j, i = np.indices((nz, n, n))
    return _index_at(s, len(s), float(F32(geom[1])), (k - nz // 2) * d, (j - n // 2) * d, (i - n // 2) * d).astype(F32)


def _ball(x):
    with np.errstate(all="ignore"):
        v = 3.0 * (np.sin(x) - x * np.cos(x)) / (x * x * x)
    return np.where(x < 1e-3, 1.0 - x * x / 10.0, v)


def _partial_waves(x, m):
    """src/phantom.cpp:44-80."""
    lmax = int(x + 4.0 * np.cbrt(x) + 10.0)

    def ratios(z):
        rho = np.zeros(lmax + 1)
        r = 0.0
        for l in range(lmax + 60, 0, -1):
            r = 1.0 / ((2.0 * l + 1.0) / z - r)
            if l <= lmax:
                rho[l] = r
        return rho

    rx, rm = ratios(x), ratios(m * x)
    c = np.zeros(lmax + 1, np.complex128)
    j_prev, j = math.cos(x) / x, math.sin(x) / x
    y_prev, y = math.sin(x) / x, -math.cos(x) / x
    for l in range(lmax + 1):
        if l > 0:
            y_next = (2.0 * l - 1.0) / x * y - y_prev
            y_prev, y = y, y_next
            j_prev, j = j, rx[l] * j
        h = complex(j, y)
        h_prev = complex(j_prev, y_prev)
        dj = j_prev - (l + 1.0) / x * j
        dh = h_prev - (l + 1.0) / x * h
        d = (1.0 / math.tan(m * x) if l == 0 else 1.0 / rm[l]) - (l + 1.0) / (m * x)
        c[l] = (m * d * j - dj) / (dh - m * d * h)
    return c


def forward_fields(spheres, illuminations, geom, n, model="rytov"):
    """src/phantom.cpp:102-191 (analytic Born / Rytov cap spectra; exact partial waves)."""
    s = np.asarray(spheres, F32).reshape(-1, 5).astype(np.float64)
    il = np.asarray(illuminations, F32).reshape(-1, 2).astype(np.float64)
    lam, nm, na, d = (float(F32(v)) for v in geom)
    k0 = 2.0 * math.pi / lam
    fm2 = nm * nm / (lam * lam)
    fna2 = na * na / (lam * lam)
    df = 1.0 / (n * d)
    if model == "exact" and len(s) != 1:
        raise ValueError("forward_fields: the exact model takes exactly one sphere")
    km = k0 * nm
    waves = _partial_waves(km * s[0, 3], s[0, 4] / nm) if model == "exact" else None
    steps = []
    for i in range(len(s)):
        parent = float(_index_at(s, i, nm, s[i, 0], s[i, 1], s[i, 2]))
        vol = 4.0 / 3.0 * math.pi * s[i, 3] ** 3
        steps.append(k0 * k0 * (s[i, 4] ** 2 - parent * parent) * vol)
    sb = signed_bin(np.arange(n), n).astype(np.float64)
    my = (sb * df)[:, None]
    mx = (sb * df)[None, :]
    ky, kx = np.indices((n, n))
    out = np.zeros((len(il), n, n), C64)
    for a in range(len(il)):
        fiy, fix = il[a]
        if fiy * fiy + fix * fix >= fm2:
            raise ValueError("forward_fields: illumination beyond n_medium / wavelength")
        fiz = math.sqrt(fm2 - fiy * fiy - fix * fix)
        fy = my + fiy
        fx = mx + fix
        rho2 = fy * fy + fx * fx
        ok = (rho2 <= fna2) & (rho2 < fm2)
        nuz = np.sqrt(np.where(ok, fm2 - rho2, 1.0))
        qz = nuz - fiz
        q = 2.0 * math.pi * np.sqrt(qz * qz + my * my + mx * mx)
        o = np.zeros((n, n), np.complex128)
        if model == "exact":
            cos_t = (fy * fiy + fx * fix + nuz * fiz) / fm2
            total = np.zeros((n, n), np.complex128)
            p_prev = np.zeros((n, n))
            p = np.ones((n, n))
            for l in range(len(waves)):
                w = 2.0 * l + 1.0
                total += w * waves[l] * p
                p_next = (w * cos_t * p - l * p_prev) / (l + 1.0)
                p_prev, p = p, p_next
            ph = -2.0 * math.pi * (qz * s[0, 0] + my * s[0, 1] + mx * s[0, 2])
            o = 4.0 * math.pi * complex(0.0, -1.0 / km) * total * np.exp(1j * ph)
        else:
            for i in range(len(s)):
                ph = -2.0 * math.pi * (qz * s[i, 0] + my * s[i, 1] + mx * s[i, 2])
                o = o + steps[i] * _ball(q * s[i, 3]) * np.exp(1j * ph)
        u = 1j / (4.0 * math.pi * nuz) * o * parity(ky + kx).astype(np.float64) / (d * d)
        out[a] = np.where(ok, u, 0.0).astype(C64)
    out = fft(out, (1, 2), False, F32(1.0) / F32(n * n))
    if model == "rytov":
        return np.exp(out.astype(np.complex128)).astype(C64)
    return (1.0 + out.astype(np.complex128)).astype(C64)


def synthesize_holograms(ratio, illuminations, geom, carrier=(5.0, 5.0), reference_amplitude=1.0, noise=0.0,
                         seed=1):
    """src/phantom.cpp:193-221, |R + u|^2 + noise. The noise samples come from numpy's generator
    seeded with `seed`, not from std::mt19937_64, so they differ from the reference's draws while
    having the same distribution; noise-free holograms agree with the reference to rounding."""
    r = np.asarray(ratio, C64)
    if r.ndim == 2:
        r = r[None]
    il = np.asarray(illuminations, F32).reshape(-1, 2).astype(np.float64)
    if r.shape[0] != il.shape[0]:
        raise ValueError("synthesize_holograms: need one illumination per field")
    nz, ny, nx = r.shape
    d = float(F32(geom[3]))
    ry = ((np.arange(ny) - ny // 2) * d)[:, None]
    rx = ((np.arange(nx) - nx // 2) * d)[None, :]
    cy, cx = float(F32(carrier[0])), float(F32(carrier[1]))
    ref = float(F32(reference_amplitude)) * np.exp(-2j * math.pi * (cy * ry + cx * rx))
    out = np.zeros(r.shape, F32)
    rng = np.random.default_rng(seed)
    for a in range(nz):
        ui = np.exp(2j * math.pi * (il[a, 0] * ry + il[a, 1] * rx))
        u = ui * r[a].astype(np.complex128)
        v = np.abs(ref + u) ** 2
        out[a] = v.astype(F32)
        if noise > 0:
            out[a] += rng.normal(0.0, float(noise), size=(ny, nx)).astype(F32)
    return out
