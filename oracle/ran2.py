"""ORACLE -- test infrastructure only.

Pure-Python restatement of the thesis's ran2 (src/random.jl:31-90) and of the
radial Thomas-Fermi sampling (src/initial.jl:161-203, 323-328), for small
cases: the product's C++ sampler is checked against it draw for draw.
Int32 wrap-around is reproduced explicitly (the generator overflows on
purpose: IQ1 reads 3668 instead of 53668).
"""
from __future__ import annotations

import math

import numpy as np

IM1, IM2 = 2147483563, 2147483399
IMM1 = IM1 - 1
IA1, IA2, IQ2, IR1, IR2 = 40014, 40692, 52774, 12211, 3791
NTAB = 32
NDIV = 1 + (IMM1 - 1) // NTAB
AM = np.float32(1) / np.float32(IM1)
RNMX = np.float32(1) - np.float32(1.2e-7)


def _i32(x: int) -> int:
    x &= 0xFFFFFFFF
    return x - (1 << 32) if x >= (1 << 31) else x


def _div(x: int, q: int) -> int:  # Julia's truncating div
    return int(x / q) if x >= 0 else -((-x) // q)


def _step(x, q, r, a, m):
    k = _div(x, q)
    x = _i32(_i32(a * _i32(x - _i32(k * q))) - _i32(k * r))
    return _i32(x + m) if x < 0 else x


class Ran2:
    def __init__(self, seed: int = -1, consistent: bool = False):
        self.iq1 = 53668 if consistent else 3668
        self.idum = max(-seed, 1)
        self.idum2 = self.idum
        self.iv = [0] * NTAB
        for j in range(NTAB + 8, 0, -1):
            self.idum = _step(self.idum, self.iq1, IR1, IA1, IM1)
            if j <= NTAB:
                self.iv[j - 1] = self.idum
        self.iy = self.iv[0]

    def next(self) -> np.float32:
        self.idum = _step(self.idum, self.iq1, IR1, IA1, IM1)
        self.idum2 = _step(self.idum2, IQ2, IR2, IA2, IM2)
        j = 1 + _div(self.iy, NDIV)
        self.iy = _i32(self.iv[j - 1] - self.idum2)
        self.iv[j - 1] = self.idum
        if self.iy < 1:
            self.iy = _i32(self.iy + IMM1)
        v = np.float32(AM * np.float32(self.iy))
        return min(v, RNMX)


def _interp_regular(v, u, n):
    j = min(math.floor(u * (n - 1)) + 1, n - 1)
    a = (j - 1) / (n - 1)
    b = j / (n - 1)
    return v[j - 1] + (v[j] - v[j - 1]) * (u - a) / (b - a)


def _on_sphere(r, uphi, umu):
    mu = 2 * umu - 1
    s = math.sqrt(1 - mu * mu)
    phi = (2 * math.pi) * uphi
    return (r * math.cos(phi) * s, r * math.sin(phi) * s, r * mu)


def sample_thomas_fermi(quantiles, density, rmax, npart, weight, seed=-1):
    rng = Ran2(seed)
    fermi = math.cbrt(3 * (math.pi * math.pi))
    nq, nr = len(quantiles), len(density)
    pos, mom = np.empty((npart, 3)), np.empty((npart, 3))
    for i in range(npart):
        x = [float(rng.next()) for _ in range(6)]
        r = _interp_regular(quantiles, x[0], nq)
        pos[i] = _on_sphere(r, x[1], x[2])
        rho = _interp_regular(density, r / rmax, nr)
        p = math.cbrt(x[3]) * fermi * math.cbrt(rho)
        mom[i] = _on_sphere(p * weight, x[4], x[5])
    return pos, mom
