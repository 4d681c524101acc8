"""Named workloads of the benchmark plan (grid sizes, radii, rules, seeds).

The single-grid workloads use the reference generator's start grid
(CPUBenchmark.cpp:21-32, CAStateGenerator.h:11-37).  The batched workload draws
every grid's parameters from a 64-bit Mersenne Twister (Matsumoto & Nishimura's
MT19937-64, default parameters, the sequence of C++ std::mt19937_64) seeded with
4, in this order per grid i:
    u  = draw / 2^64           side  n = round(64 * 32^u)      (log-uniform on [64, 2048])
    R  = 1 + draw % 8          radius uniform on {1..8}
    v  = draw / 2^64           density d = 0.2 + 0.4 v          (uniform on [0.2, 0.6])
and the grid's cells come from the reference generator with state seed
(4 * 1000003 + 7919 * i) % 1000000 and one generator thread.  The rule is the
interval rule scaled to N = (2R+1)^2 (see scaled_rule).
"""

MASK64 = (1 << 64) - 1


class MT19937_64:
    """MT19937-64 (Matsumoto & Nishimura), same output sequence as std::mt19937_64."""

    def __init__(self, seed):
        self.mt = [0] * 312
        self.mt[0] = seed & MASK64
        for i in range(1, 312):
            prev = self.mt[i - 1]
            self.mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) & MASK64
        self.idx = 312

    def _twist(self):
        mt = self.mt
        for i in range(312):
            x = (mt[i] & 0xFFFFFFFF80000000) | (mt[(i + 1) % 312] & 0x7FFFFFFF)
            xa = x >> 1
            if x & 1:
                xa ^= 0xB5026F5AA96619E9
            mt[i] = mt[(i + 156) % 312] ^ xa
        self.idx = 0

    def __call__(self):
        if self.idx >= 312:
            self._twist()
        y = self.mt[self.idx]
        self.idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & MASK64


def scaled_rule(radius):
    """Interval rule scaled to N=(2R+1)^2, centre counted: birth [ceil(0.34N), floor(0.45N)],
    survival [ceil(0.33N), floor(0.57N)]; returned in the reference's centre-excluded
    convention (survival bounds - 1), integer arithmetic."""
    N = (2 * radius + 1) ** 2
    bmin, bmax = -((-34 * N) // 100), (45 * N) // 100
    smin, smax = -((-33 * N) // 100) - 1, (57 * N) // 100 - 1
    return (smin, smax, bmin, bmax)


BOSCO_R5 = (32, 56, 34, 45)


def batch_config(count=4096, seed=4):
    """[(n, R, rule, density, state_seed)] for the batched workload."""
    rng = MT19937_64(seed)
    out = []
    for i in range(count):
        u = rng() / 2.0 ** 64
        n = int(round(64 * 32.0 ** u))
        n = max(64, min(2048, n))
        r = 1 + rng() % 8
        d = 0.2 + 0.4 * (rng() / 2.0 ** 64)
        state_seed = (seed * 1000003 + 7919 * i) % 1000000
        out.append((n, r, scaled_rule(r), d, state_seed))
    return out
