"""``java.util.Random``, the documented 48-bit linear congruential generator of the Java SE API.

The reference's tests draw every randomised fixture from ``new java.util.Random(seed)``; this port reproduces
those fixtures exactly (``nextDouble`` = ``((next(26) << 27) + next(27)) * 2**-53``).
"""

_MULTIPLIER = 0x5DEECE66D
_ADDEND = 0xB
_MASK = (1 << 48) - 1


class JavaRandom:
    def __init__(self, seed: int):
        self.seed = (seed ^ _MULTIPLIER) & _MASK

    def next(self, bits: int) -> int:
        self.seed = (self.seed * _MULTIPLIER + _ADDEND) & _MASK
        r = self.seed >> (48 - bits)
        if r >= 1 << (bits - 1) and bits == 32:
            r -= 1 << 32
        return r

    def next_double(self) -> float:
        return ((self.next(26) << 27) + self.next(27)) * (1.0 / (1 << 53))

    def next_int(self) -> int:
        return self.next(32)
