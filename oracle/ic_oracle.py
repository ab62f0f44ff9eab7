"""CPU restatement (numpy, float64) of gadget-ng's Zel'dovich initial conditions.

Test infrastructure only.  Follows
  crates/gadget-ng-core/src/transfer_fn.rs:89-127 (Eisenstein-Hu no-wiggle
    T(k)), :146-184 (sigma^2(R) trapezoid in ln k, 8192 steps over
    [1e-5, 5e2] h/Mpc), :190-199 (top-hat window), :222-228 (amplitude for
    sigma_8);
  crates/gadget-ng-core/src/ic_zeldovich.rs:387-466 (sigma(|n|) per mode:
    power law A |n|^(n_s/4) / sqrt(N^3), Eisenstein-Hu A k^(n_s/2) T(k) /
    sqrt(N^3) with k = 2 pi |n| h / L_h), :287-371 (Gaussian modes, DC and
    Nyquist planes zero, Hermitian pairs), :541-616 (Psi(k) = i n / |n|^2
    delta(k), inverse FFT, times cell / N^3), :686-760 (lattice at cell
    centres + Psi wrapped, momentum a^2 f H Psi, optional D(a)/D(1) rescale);
  crates/gadget-ng-core/src/cosmology.rs:509-520 (H(a), LCDM), :598-610
    (f = Omega_m(a)^0.55), :650-666 and :736-742 (CPT92 growth ratio).
Per-mode seeds are the reference's mode_seed (ic_zeldovich.rs:27-42: murmur3
fmix64 of seed ^ fmix64(ix n^2 + iy n + iz)).  The reference then draws two
uniforms from rand::StdRng (ChaCha12, rand 0.10.1 / chacha20 0.10.0, crates
absent here) seeded by that value; this restatement and the device draw them
from SplitMix64 seeded there instead, so their realisations agree with each
other value for value and with the reference's in distribution only.
Parity of the realisation with the reference is unpinned; its normalisation
is pinned by the reference's committed rms(Psi) and v_rms figures.
"""
from __future__ import annotations

import math

import numpy as np


def transfer_eh_nowiggle(k_hmpc, omega_m, omega_b, h):
    k = np.asarray(k_hmpc, dtype=np.float64)
    om_h2 = omega_m * h * h
    ob_h2 = omega_b * h * h
    fb = omega_b / omega_m
    s = 44.5 * math.log(9.83 / om_h2) / math.sqrt(1.0 + 10.0 * ob_h2 ** 0.75)
    ag = 1.0 - 0.328 * math.log(431.0 * om_h2) * fb + 0.38 * math.log(22.3 * om_h2) * fb * fb
    ks = 0.43 * (k * h) * s
    gamma = omega_m * h * (ag + (1.0 - ag) / (1.0 + ks ** 4))
    q = k / np.maximum(gamma, 1e-30)
    l0 = np.log(math.e * 2.0 + 1.8 * q)
    c0 = 14.2 + 731.0 / (1.0 + 62.5 * q)
    t = np.clip(l0 / (l0 + c0 * q * q), 0.0, 1.0)
    return np.where(k <= 0.0, 1.0, t)


def tophat(x):
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        w = 3.0 * (np.sin(x) - x * np.cos(x)) / (x * x * x)
    return np.where(np.abs(x) < 1e-4, 1.0 - x * x / 10.0, w)


def sigma_sq_unit(r, n_s, omega_m, omega_b, h):
    lk0, lk1, steps = math.log(1e-5), math.log(5e2), 8192
    dl = (lk1 - lk0) / steps
    k = np.exp(lk0 + np.arange(steps + 1) * dl)
    k[0] = 1e-5
    t = transfer_eh_nowiggle(k, omega_m, omega_b, h)
    w = tophat(k * r)
    f = k ** (n_s + 3.0) * t * t * w * w
    s = 0.0
    for i in range(1, steps + 1):  # the reference's running trapezoid
        s += 0.5 * (f[i - 1] + f[i]) * dl
    return s / (2.0 * math.pi * math.pi)


def amplitude_for_sigma8(sigma8, n_s, omega_m, omega_b, h):
    v = sigma_sq_unit(8.0, n_s, omega_m, omega_b, h)
    return sigma8 if v <= 0.0 else sigma8 / math.sqrt(v)


def sigma_of_n(n_abs, n, kind, amplitude, n_s, omega_m=0.31, omega_b=0.049, h=0.68, box_mpc_h=100.0,
               sigma8=None):
    """Per-mode standard deviation sigma(|n|) of the reference's spectrum closure."""
    n_abs = np.asarray(n_abs, dtype=np.float64)
    inv = 1.0 / math.sqrt(float(n) ** 3)
    if kind == "power_law":
        with np.errstate(divide="ignore"):
            return np.where(n_abs <= 0.0, 0.0, amplitude * n_abs ** (n_s / 4.0) * inv)
    amp = amplitude_for_sigma8(sigma8, n_s, omega_m, omega_b, h) if sigma8 else amplitude
    k = 2.0 * math.pi * h / box_mpc_h * n_abs
    with np.errstate(divide="ignore", invalid="ignore"):
        v = amp * k ** (n_s / 2.0) * transfer_eh_nowiggle(k, omega_m, omega_b, h) * inv
    return np.where(n_abs <= 0.0, 0.0, v)


def hubble(a, omega_m, omega_l, h0):
    return h0 * math.sqrt(max(omega_m / (a * a * a) + omega_l, 0.0))


def growth_rate_f(a, omega_m, omega_l, h0):
    hh = hubble(a, omega_m, omega_l, h0)
    om_a = omega_m / (a * a * a) / ((hh / h0) ** 2)
    return max(om_a, 0.0) ** 0.55


def growth_d(a, omega_m, omega_l):
    a3 = a * a * a
    den = omega_m + omega_l * a3
    om, ol = omega_m / den, omega_l * a3 / den
    br = max(om, 0.0) ** (4.0 / 7.0) - ol + (1.0 + om / 2.0) * (1.0 + ol / 70.0)
    return a * 2.5 * om / br


def mode_int(n):
    j = np.arange(n)
    return np.where(j <= n // 2, j, j - n)


def expected_psi2(n, box, sig):
    """E[<|Psi|^2>] over the lattice for per-mode sigma sig[ix, iy, iz]."""
    f = mode_int(n).astype(np.float64)
    nx, ny, nz = np.meshgrid(f, f, f, indexing="ij")
    n2 = nx * nx + ny * ny + nz * nz
    half = n // 2
    keep = (n2 > 0) & (np.abs(nx) != half) & (np.abs(ny) != half) & (np.abs(nz) != half)
    d = box / n
    return float((d / n ** 3) ** 2 * np.sum(2.0 * sig[keep] ** 2 / n2[keep]))


_M64 = np.uint64


def fmix64(x):
    """Murmur3 64-bit finalizer, the reference's hash_u64 (ic_zeldovich.rs:27-35)."""
    x = np.array(x, dtype=np.uint64, copy=True)
    x ^= x >> _M64(33)
    x *= _M64(0xFF51AFD7ED558CCD)
    x ^= x >> _M64(33)
    x *= _M64(0xC4CEB9FE1A85EC53)
    x ^= x >> _M64(33)
    return x


def splitmix64(state, count):
    """The first `count` outputs of SplitMix64 (Steele, Lea and Flood 2014) per seed."""
    st = np.array(state, dtype=np.uint64, copy=True)
    out = []
    for _ in range(count):
        st = st + _M64(0x9E3779B97F4A7C15)
        z = st.copy()
        z = (z ^ (z >> _M64(30))) * _M64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> _M64(27))) * _M64(0x94D049BB133111EB)
        out.append(z ^ (z >> _M64(31)))
    return out


def gaussian_std(seed):
    """Box-Muller on two uniforms of 53 bits (ic_zeldovich.rs:45-57), stream SplitMix64."""
    a, b = splitmix64(seed, 2)
    u1 = np.maximum((a >> _M64(11)).astype(np.float64) / 9007199254740992.0, 1e-300)
    u2 = (b >> _M64(11)).astype(np.float64) / 9007199254740992.0
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def _modes(n):
    f = mode_int(n)
    nx, ny, nz = np.meshgrid(f, f, f, indexing="ij")
    n2 = (nx * nx + ny * ny + nz * nz).astype(np.float64)
    half = n // 2
    keep = (n2 > 0) & (np.abs(nx) != half) & (np.abs(ny) != half) & (np.abs(nz) != half)
    return (nx, ny, nz), n2, keep


def delta_kspace(n, seed, sig):
    """generate_delta_kspace (ic_zeldovich.rs:287-385), indexed [ix, iy, iz]:
    every mode draws from its own mode_seed, then for each pair {k, -k} the one
    with the larger packed index takes the conjugate of the other."""
    i = np.arange(n)
    ix, iy, iz = np.meshgrid(i, i, i, indexing="ij")
    packed = (ix * n * n + iy * n + iz).astype(np.uint64)
    ms = fmix64(_M64(seed) ^ fmix64(packed))
    g_r = gaussian_std(ms)
    g_i = gaussian_std(fmix64(ms ^ _M64(0x9E3779B97F4A7C15)))
    _, _, keep = _modes(n)
    delta = np.where(keep, sig * g_r + 1j * (sig * g_i), 0.0)
    neg = (-i) % n
    twin_packed = (neg[ix] * n * n + neg[iy] * n + neg[iz]).astype(np.uint64)
    conj_twin = np.conj(delta[neg[ix], neg[iy], neg[iz]])
    return np.where((packed < twin_packed) | ~keep, delta, conj_twin)


def displacement(delta, n, box):
    """delta_to_displacement (ic_zeldovich.rs:541-616): Psi_a = Re(IFFT(i n_a /
    |n|^2 delta)) / n^3 * cell, and the largest |Im| of the three transforms."""
    comps, n2, _ = _modes(n)
    d = box / n
    psi, max_im = [], 0.0
    for comp in comps:
        with np.errstate(invalid="ignore", divide="ignore"):
            ph = np.where(n2 > 0, 1j * comp / n2 * delta, 0.0)
        c = np.fft.ifftn(ph) * (n ** 3)  # unnormalised inverse, as rustfft's
        max_im = max(max_im, float(np.max(np.abs(c.imag))))
        psi.append(c.real / n ** 3 * d)
    return psi, max_im


def zeldovich(n, box, sig, seed=0, vel_factor=1.0, scale=1.0):
    """Positions (N, 3) and momenta of the realisation the device generates for
    `seed` (zeldovich_ics, ic_zeldovich.rs:686-760): gid = ix n^2 + iy n + iz,
    x = (i + 1/2) cell + scale Psi wrapped into [0, box), p = vel_factor scale Psi."""
    psi, _ = displacement(delta_kspace(n, seed, sig), n, box)
    psi = [p * scale for p in psi]
    d = box / n
    g = (np.arange(n) + 0.5) * d
    qx, qy, qz = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([(qx + psi[0]) % box, (qy + psi[1]) % box, (qz + psi[2]) % box], -1).reshape(-1, 3)
    mom = np.stack(psi, -1).reshape(-1, 3) * vel_factor
    return pos, mom


# ---- second order (crates/gadget-ng-core/src/ic_2lpt.rs) -------------------------
def phi_second_derivatives(delta, n):
    """phi_ab = Re(IFFT(-n_a n_b / |n|^2 delta)) / n^3 for ab = xx, yy, zz, xy,
    xz, yz (ic_2lpt.rs:86-140)."""
    (nx, ny, nz), n2, _ = _modes(n)
    comps = (nx, ny, nz)
    out = []
    for a, b in ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)):
        with np.errstate(invalid="ignore", divide="ignore"):
            ph = np.where(n2 > 0, -comps[a] * comps[b] / n2 * delta, 0.0)
        out.append(np.fft.ifftn(ph).real)  # ifftn divides by n^3, as the reference's ifft_norm
    return out


def source_2lpt(d):
    """S = (xx yy - xy^2) + (yy zz - yz^2) + (zz xx - xz^2) (ic_2lpt.rs:146-165)."""
    xx, yy, zz, xy, xz, yz = d
    return (xx * yy - xy * xy) + (yy * zz - yz * yz) + (zz * xx - xz * xz)


def source_to_psi2(s, n, box):
    """Psi2_a = Re(IFFT(-i n_a / |n|^2 FFT(S))) / n^3 * cell, zero at DC and on
    the Nyquist planes (ic_2lpt.rs:181-240)."""
    (nx, ny, nz), n2, keep = _modes(n)
    sk = np.fft.fftn(s)
    d = box / n
    out = []
    for comp in (nx, ny, nz):
        with np.errstate(invalid="ignore", divide="ignore"):
            ph = np.where(keep, -1j * comp / n2 * sk, 0.0)
        out.append(np.fft.ifftn(ph).real * d)
    return out


def lpt_factors(a_init=1.0, omega_m=1.0, omega_l=0.0, h0=1.0, cosmology=False):
    """(a^2 f1 H, D2/D1^2, a^2 f2 H D2/D1^2) of ic_2lpt.rs:404-446; without
    cosmology a = 1, Omega_m = 1, Omega_L = 0."""
    a, om, ol = (a_init, omega_m, omega_l) if cosmology else (1.0, 1.0, 0.0)
    hh = hubble(a, om, ol, h0)
    om_a = max(om / a ** 3 / (hh / h0) ** 2, 0.0)
    f1 = om_a ** 0.55
    f2 = 2.0 * om_a ** (6.0 / 11.0)
    d21 = -3.0 / 7.0 * om_a ** (-1.0 / 143.0)
    return a * a * f1 * hh, d21, a * a * f2 * hh * d21


def zeldovich_2lpt(n, box, sig, seed=0, vel1=1.0, d21=-3.0 / 7.0, vel2=-6.0 / 7.0, scale=1.0):
    """zeldovich_2lpt_ics (ic_2lpt.rs:386-550) on the realisation of `seed`:
    x = q + scale Psi1 + d21 scale^2 Psi2 wrapped, p = vel1 scale Psi1 + vel2
    scale^2 Psi2.  Returns positions, momenta and the scaled Psi2."""
    delta = delta_kspace(n, seed, sig)
    psi1, _ = displacement(delta, n, box)
    psi2 = source_to_psi2(source_2lpt(phi_second_derivatives(delta, n)), n, box)
    d = box / n
    g = (np.arange(n) + 0.5) * d
    qx, qy, qz = np.meshgrid(g, g, g, indexing="ij")
    s1 = [p * scale for p in psi1]
    s2 = [p * scale * scale for p in psi2]
    pos = np.stack([(q + a + d21 * b) % box for q, a, b in zip((qx, qy, qz), s1, s2)], -1).reshape(-1, 3)
    mom = np.stack([vel1 * a + vel2 * b for a, b in zip(s1, s2)], -1).reshape(-1, 3)
    return pos, mom, np.stack(s2, -1).reshape(-1, 3)
