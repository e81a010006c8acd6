"""CPU restatement of HYOWON's generated initial conditions (TEST
INFRASTRUCTURE ONLY; the checker for hyowon_ic_field / hyowon_ic_generate /
hyowon_pm_generate_ics). Only tests/ import it.

* Philox4x32-10 (src/ic/philox_rng.cpp:43-62): per round the 32x32->64
  products of counter words 0 and 2 with the two multipliers, the new counter
  (hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0), the key bumped by the two Weyl
  constants between rounds. The counter of a mode is (kx, ky, kz, stream) as
  u32 words, the key the seed's low and high words (:64-83).
* 53-bit open uniforms (:27-36): bits = (w_hi << 21) | (w_lo >> 11), u = bits
  2^-53, or 2^-54 when bits == 0. Box-Muller (:85-96): r = sqrt(-2 ln u1),
  theta = 2 pi u2, (r cos theta, r sin theta). math.log / math.cos /
  math.sin are the C library's, as in the reference build.
* The mode loop of RandomField::generate (src/ic/random_field.cpp:70-330):
  k = 0 and modes outside the Cartesian support |m_i| <= K are zero;
  on the kz = 0 and Nyquist planes the mode whose conjugate (N-i, N-j) is
  smaller (i first, then j) is drawn from the conjugate's counter and its
  imaginary part negated; self-conjugate modes take sqrt(var) n1 (gaussian)
  or +-sqrt(var) by u1 < 0.5 (fixed); the others sqrt(var/2) (n1, n2)
  (gaussian) or sqrt(var) e^{2 pi i u1} (fixed, stream 1); pair_b negates
  every mode. var = M^6/L^3 P(sqrt(|m|^2) k_f) formed as
  math::ScaledPositiveProduct (include/cosmo_nbody/math/scaled_positive_product.hpp:
  425-512): long-double mantissa/exponent, one factor at a time.
* LPTDisplacement::apply_to_arrays (src/ic/lpt_displacement.cpp:150-520):
  psi1_k = (-Im d, Re d) k_a / k^2 (k_a = 0 on axis a's Nyquist plane),
  c2r * 1/M^3, sampled at lattice node (i, j, k) * M/N, x = wrap(q + psi),
  p = p1 psi; for 2LPT the source
  S = -1/2 sum_a H_aa^2 - sum_{a<b} H_ab^2 + 1/2 (tr H)^2 with
  H_ab = c2r(d k_a k_b / k^2) (mixed terms 0 on either Nyquist plane) and
  tr H = c2r(d) (k = 0 removed), accumulated in that order; r2c of S,
  Cartesian band limit |m_i| <= K (src/ic/particle_lattice_bandlimit.cpp:42-80),
  psi2_k = (Im S, -Re S) k_a / k^2, x += x2 psi2, p += p2 psi2.
  Wavenumbers are (2 pi m) / L (include/cosmo_nbody/mesh/mesh_geometry.hpp:112-115).

numpy's FFT is unnormalised forward / 1/n inverse like the reference's FFT
backend; only FFT rounding separates the LPT restatement from the reference.
"""
from __future__ import annotations

import math

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(counters, keys):
    """Vectorised Philox4x32-10: counters (n, 4), keys (n, 2) -> (n, 4) uint32."""
    c = np.asarray(counters, dtype=np.uint64).reshape(-1, 4).copy()
    k = np.asarray(keys, dtype=np.uint64).reshape(-1, 2).copy()
    for r in range(10):
        p0 = np.uint64(M0) * c[:, 0]
        p1 = np.uint64(M1) * c[:, 2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & np.uint64(MASK)
        hi1, lo1 = p1 >> np.uint64(32), p1 & np.uint64(MASK)
        c = np.stack([hi1 ^ c[:, 1] ^ k[:, 0], lo1, hi0 ^ c[:, 3] ^ k[:, 1], lo0], axis=1)
        if r != 9:
            k[:, 0] = (k[:, 0] + np.uint64(W0)) & np.uint64(MASK)
            k[:, 1] = (k[:, 1] + np.uint64(W1)) & np.uint64(MASK)
    return c.astype(np.uint32)


def _open_uniform(hi, lo):
    bits = (hi.astype(np.uint64) << np.uint64(21)) | (lo.astype(np.uint64) >> np.uint64(11))
    u = bits.astype(np.float64) * 2.0 ** -53
    return np.where(bits == 0, 2.0 ** -54, u)


def mode_draws(seed, stream, modes):
    """(u1, u2, n1, n2) per integer mode (n, 3) -- uniform_pair_open01 and
    normal_pair of src/ic/philox_rng.cpp:64-96."""
    m = np.asarray(modes, dtype=np.int64).reshape(-1, 3)
    ctr = np.empty((m.shape[0], 4), dtype=np.uint64)
    ctr[:, :3] = m & MASK
    ctr[:, 3] = stream
    key = np.empty((m.shape[0], 2), dtype=np.uint64)
    key[:, 0] = seed & MASK
    key[:, 1] = (seed >> 32) & MASK
    w = philox4x32_10(ctr, key)
    u1 = _open_uniform(w[:, 0], w[:, 1])
    u2 = _open_uniform(w[:, 2], w[:, 3])
    r = np.array([math.sqrt(-2.0 * math.log(v)) for v in u1])
    th = 2.0 * math.pi * u2
    n1 = r * np.array([math.cos(v) for v in th])
    n2 = r * np.array([math.sin(v) for v in th])
    return np.stack([u1, u2, n1, n2], axis=1)


def _consume(mant, expo, factor, divide):
    fm, fe = np.frexp(np.float64(factor))
    fw = np.longdouble(fm)
    if divide:
        mant = mant / fw
        expo -= int(fe)
    else:
        mant = mant * fw
        expo += int(fe)
    mant, ne = np.frexp(mant)
    return mant, expo + int(ne)


def mode_amplitudes(M: int, L: float, power):
    """(s, 2) table {sqrt(var_s), sqrt(var_s / 2)} for var_s = M^6 / L^3 P_s,
    formed like ScaledPositiveProduct::from_quotient(...).multiplied_by(P_s)
    (ordinary range only); s = 0 gives zeros."""
    mant, expo = np.longdouble(1.0), 0
    for _ in range(6):
        mant, expo = _consume(mant, expo, float(M), False)
    for _ in range(3):
        mant, expo = _consume(mant, expo, float(L), True)
    power = np.asarray(power, dtype=np.float64)
    out = np.zeros((power.size, 2))
    for s in range(1, power.size):
        m2, e2 = _consume(mant, expo, power[s], False)
        var = float(np.ldexp(m2, e2))
        out[s, 0] = math.sqrt(var)
        out[s, 1] = math.sqrt(var / 2.0)
    return out


def represented_wavenumbers(L: float, K: int):
    """k_s = double(sqrt(long double s)) * (2 pi / L), s = 0 .. 3K^2
    (include/cosmo_nbody/ic/particle_lattice_bandlimit.hpp:27-37)."""
    s = np.arange(3 * K * K + 1, dtype=np.longdouble)
    return np.sqrt(s).astype(np.float64) * (2.0 * math.pi / L)


def _mode_numbers(n):
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n)


def gaussian_field(M: int, seed: int, K: int, amp, fixed=False, pairing=0):
    """RandomField::generate on an M^3 mesh, half spectrum (M, M, M/2+1)."""
    amp = np.asarray(amp, dtype=np.float64)
    Hz = M // 2 + 1
    I, J, Kz = np.meshgrid(np.arange(M), np.arange(M), np.arange(Hz), indexing="ij")
    I, J, Kz = I.ravel(), J.ravel(), Kz.ravel()
    mx, my = _mode_numbers(M)[I], _mode_numbers(M)[J]
    mz = Kz.astype(np.int64)
    inside = (np.abs(mx) <= K) & (np.abs(my) <= K) & (mz <= K) & ((mx != 0) | (my != 0) | (mz != 0))
    plane = (Kz == 0) | ((M % 2 == 0) & (Kz == M // 2))
    ci, cj = (M - I) % M, (M - J) % M
    selfc = plane & (ci == I) & (cj == J)
    conj = plane & ~selfc & ((ci < I) | ((ci == I) & (cj < J)))
    ui = np.where(conj, ci, I)
    uj = np.where(conj, cj, J)
    cx, cy = _mode_numbers(M)[ui], _mode_numbers(M)[uj]
    s = mx * mx + my * my + mz * mz
    out = np.zeros(I.size, dtype=np.complex128)
    sel = np.nonzero(inside)[0]
    d = mode_draws(seed, 1 if fixed else 0, np.stack([cx[sel], cy[sel], mz[sel]], axis=1))
    a1, a2 = amp[s[sel], 0], amp[s[sel], 1]
    sc, cj_ = selfc[sel], conj[sel]
    if fixed:
        ph = 2.0 * math.pi * d[:, 0]
        im = a1 * np.array([math.sin(v) for v in ph])
        re = a1 * np.array([math.cos(v) for v in ph])
        re = np.where(sc, np.where(d[:, 0] < 0.5, -a1, a1), re)
        im = np.where(sc, 0.0, np.where(cj_, -im, im))
    else:
        re = np.where(sc, a1 * d[:, 2], a2 * d[:, 2])
        im = np.where(sc, 0.0, np.where(cj_, -(a2 * d[:, 3]), a2 * d[:, 3]))
    v = re + 1j * im
    if pairing == 2:
        v = -v
    out[sel] = v
    return out.reshape(M, M, Hz)


def _k_components(M, L):
    m = _mode_numbers(M).astype(np.float64)
    return 2.0 * math.pi * m / L


def _wrap(x, L):
    x = np.asarray(x, dtype=np.float64)
    inside = (x >= 0.0) & (x < L)
    w = np.fmod(x, L)
    w = np.where(w < 0.0, w + L, w)
    w = np.where(w >= L, 0.0, w)
    return np.where(inside, x, w)


def lpt(delta, N: int, L: float, K: int, p1: float, order=1, x2=0.0, p2=0.0):
    """LPTDisplacement::apply_to_arrays on the corner lattice; delta is the
    (M, M, M/2+1) field. Returns {x, y, z, px, py, pz} in particle order."""
    M = delta.shape[0]
    r = M // N
    kc = _k_components(M, L)
    KX = kc[:, None, None]
    KY = kc[None, :, None]
    KZ = kc[: M // 2 + 1][None, None, :]
    k2 = KX * KX + KY * KY + KZ * KZ
    nyq = [np.zeros(M, bool) for _ in range(3)]
    if M % 2 == 0:
        for a in range(3):
            nyq[a][M // 2] = True
    NYQ = [nyq[0][:, None, None], nyq[1][None, :, None], nyq[2][: M // 2 + 1][None, None, :]]
    kfull = [KX, KY, KZ]
    zero = k2 == 0.0
    safe_k2 = np.where(zero, 1.0, k2)
    inv = 1.0 / float(M) ** 3

    def c2r(f):
        return np.fft.irfftn(f, s=(M, M, M), axes=(0, 1, 2), norm="forward") * inv

    i, j, k = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    dx = L / N
    pos = [(i * dx).ravel(), (j * dx).ravel(), (k * dx).ravel()]
    mom = [np.zeros(N ** 3) for _ in range(3)]

    def apply(field_k, pf, xf):
        for a in range(3):
            kd = np.where(NYQ[a], 0.0, kfull[a])
            f = np.where(zero, 0.0, kd / safe_k2)
            psi_k = np.where(zero, 0.0, -field_k.imag * f + 1j * (field_k.real * f))
            psi = c2r(psi_k)[::r, ::r, ::r].ravel()
            disp = xf * psi
            pos[a] = _wrap(pos[a] + disp, L)
            mom[a] = mom[a] + pf * psi

    apply(delta, p1, 1.0)
    if order == 2:
        def hess(a, b):
            num = kfull[a] * kfull[b]
            if a != b:
                num = np.where(NYQ[a] | NYQ[b], 0.0, num)
            h = np.where(zero, 0.0, delta * (num / safe_k2))
            return c2r(h)
        src = None
        for a in range(3):
            h = hess(a, a)
            t = 0.5 * h * h
            src = -t if src is None else src - t
        for a, b in ((0, 1), (0, 2), (1, 2)):
            h = hess(a, b)
            src = src - h * h
        d0 = delta.copy()
        d0[0, 0, 0] = 0.0
        tr = c2r(d0)
        src = src + 0.5 * tr * tr
        S = np.fft.rfftn(src)
        m = _mode_numbers(M)
        keep = (np.abs(m)[:, None, None] <= K) & (np.abs(m)[None, :, None] <= K) \
            & (np.abs(m[: M // 2 + 1])[None, None, :] <= K)
        S = np.where(keep, S, 0.0)
        # psi2_k = (Im S, -Re S) f = -(-Im S, Re S) f: the 1LPT operator on -S
        apply(-S, p2, x2)
    return dict(x=pos[0], y=pos[1], z=pos[2], px=mom[0], py=mom[1], pz=mom[2])
