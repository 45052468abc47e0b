"""Minimal host-side Fp2 value type used when TruePix's own `libTruePix.extfield`
is not importable.

Same attributes and constructors as the reference type
(TruePix-main/libTruePix/extfield.py:29-185: `real`, `imag`, `p`; `_raw` builds
from reduced coordinates), so values returned by the bridge compare and pickle
the same way. Only the arithmetic the bridge and the tests need is provided.
"""
from __future__ import annotations

BASE_PRIME_61 = (1 << 61) - 1


class Fp2:
    __slots__ = ("real", "imag", "p")

    def __init__(self, real: int, imag: int = 0, p: int = BASE_PRIME_61):
        self.real = real % p
        self.imag = imag % p
        self.p = p

    def __getstate__(self):
        return (self.real, self.imag, self.p)

    def __setstate__(self, state):
        self.real, self.imag, self.p = state

    def __eq__(self, other):
        if isinstance(other, Fp2):
            return (self.real, self.imag, self.p) == (other.real, other.imag, other.p)
        if isinstance(other, int):
            return self.imag == 0 and self.real == other % self.p
        return NotImplemented

    def __hash__(self):
        return hash((self.real, self.imag))

    def __add__(self, o):
        o = _as(o, self.p)
        return _raw((self.real + o.real) % self.p, (self.imag + o.imag) % self.p, self.p)

    __radd__ = __add__

    def __sub__(self, o):
        o = _as(o, self.p)
        return _raw((self.real - o.real) % self.p, (self.imag - o.imag) % self.p, self.p)

    def __rsub__(self, o):
        return _as(o, self.p) - self

    def __mul__(self, o):
        o = _as(o, self.p)
        a, b, c, d, p = self.real, self.imag, o.real, o.imag, self.p
        return _raw((a * c - b * d) % p, (a * d + b * c) % p, p)

    __rmul__ = __mul__

    def __repr__(self):
        return f"Fp2({self.real}, {self.imag})"


def _raw(real: int, imag: int, p: int = BASE_PRIME_61) -> Fp2:
    v = Fp2.__new__(Fp2)
    v.real = real
    v.imag = imag
    v.p = p
    return v


def _as(x, p) -> Fp2:
    if isinstance(x, Fp2):
        return x
    return _raw(int(x) % p, 0, p)
