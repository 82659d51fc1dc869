"""ORACLE -- test infrastructure only.

The sequence of glibc's rand() with its default seed (1), restated from the published
description of glibc's additive feedback generator (the TYPE_3 state of random_r: 34
seeded words, r[i] = r[i-31] + r[i-3] mod 2^32, the first 310 values discarded, each output
r >> 1).  The reference's ID sampling draws `rand() % n` (matroxTest-V1/compression.h:641,
745); with this sequence and one thread, this repository's producer repeats those draws.
"""


class GlibcRand:
    def __init__(self, seed: int = 1):
        r = [0] * 34
        r[0] = seed & 0xFFFFFFFF
        for i in range(1, 31):
            r[i] = (16807 * r[i - 1]) % 2147483647
        for i in range(31, 34):
            r[i] = r[i - 31]
        self.r = r
        for _ in range(310):
            self._next()

    def _next(self) -> int:
        r = self.r
        v = (r[-31] + r[-3]) & 0xFFFFFFFF
        r.append(v)
        if len(r) > 64:
            del r[:-34]
        return v

    def __call__(self) -> int:
        return self._next() >> 1
