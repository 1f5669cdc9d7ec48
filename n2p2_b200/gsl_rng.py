"""The two GSL random number generators the reference's training program draws
from, restated from their published algorithms.

Reference use (src/libnnptrain): Dataset::setupRandomNumberGenerator
(Dataset.cpp:110-163) seeds rank 0's generator `rng` as gsl_rng_mt19937 with
`random_seed` and the global generator `rngGlobal` as gsl_rng_taus with the
first draw of `rng`; distributeStructures draws gsl_rng_uniform_int(rng,
numProcs) per structure (:810), Training::selectSets gsl_rng_uniform(rng) per
structure (Training.cpp:109), randomizeNeuralNetworkWeights
gsl_rng_uniform(rngGlobal) per connection (:3643), and setupTraining seeds the
two std::mt19937_64 shuffle generators with gsl_rng_get of each (:1041-1042).

* Mt19937 -- M. Matsumoto and T. Nishimura, "Mersenne Twister: a
  623-dimensionally equidistributed uniform pseudorandom number generator",
  ACM TOMACS 8 (1998) 3-30, with the authors' 2002 initialisation
  (x_i = 1812433253 (x_{i-1} xor (x_{i-1} >> 30)) + i); GSL maps seed 0 to
  4357.  Outputs 32-bit integers.
* Taus -- P. L'Ecuyer, "Maximally equidistributed combined Tausworthe
  generators", Math. Comp. 65 (1996) 203-213 (the three-component generator
  with parameters (31, 13, 12, 19), (29, 2, 4, 25), (28, 3, 17, 11)); GSL
  seeds its components with the linear congruential map s -> 69069 s mod
  2^32 (seed 0 -> 1) and discards six outputs.

uniform() is get() / 2^32 (both generators span [0, 2^32)); uniform_int(n)
divides the range into n equal bins of size floor((2^32 - 1) / n) and
redraws outputs past the last full bin.
"""

_MASK = 0xFFFFFFFF


class Mt19937:
    N = 624
    M = 397

    def __init__(self, seed):
        s = int(seed) & 0xFFFFFFFFFFFFFFFF
        if s == 0:
            s = 4357
        mt = [0] * self.N
        mt[0] = s & _MASK
        for i in range(1, self.N):
            mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & _MASK
        self._mt = mt
        self._i = self.N

    def _twist(self):
        mt, N, M = self._mt, self.N, self.M
        for i in range(N):
            y = (mt[i] & 0x80000000) | (mt[(i + 1) % N] & 0x7FFFFFFF)
            v = mt[(i + M) % N] ^ (y >> 1)
            if y & 1:
                v ^= 0x9908B0DF
            mt[i] = v
        self._i = 0

    def get(self):
        if self._i >= self.N:
            self._twist()
        y = self._mt[self._i]
        self._i += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & _MASK

    def uniform(self):
        return self.get() / 4294967296.0

    def uniform_int(self, n):
        return _uniform_int(self, n)


class Taus:
    def __init__(self, seed):
        s = int(seed) & 0xFFFFFFFFFFFFFFFF
        if s == 0:
            s = 1
        self.s1 = (69069 * s) & _MASK
        self.s2 = (69069 * self.s1) & _MASK
        self.s3 = (69069 * self.s2) & _MASK
        for _ in range(6):
            self.get()

    def get(self):
        s1, s2, s3 = self.s1, self.s2, self.s3
        s1 = (((s1 & 4294967294) << 12) & _MASK) ^ ((((s1 << 13) & _MASK) ^ s1) >> 19)
        s2 = (((s2 & 4294967288) << 4) & _MASK) ^ ((((s2 << 2) & _MASK) ^ s2) >> 25)
        s3 = (((s3 & 4294967280) << 17) & _MASK) ^ ((((s3 << 3) & _MASK) ^ s3) >> 11)
        self.s1, self.s2, self.s3 = s1, s2, s3
        return s1 ^ s2 ^ s3

    def uniform(self):
        return self.get() / 4294967296.0

    def uniform_int(self, n):
        return _uniform_int(self, n)


def _uniform_int(gen, n):
    n = int(n)
    if n <= 0 or n > _MASK:
        raise ValueError("n must be in [1, 2^32 - 1]")
    scale = _MASK // n
    while True:
        k = gen.get() // scale
        if k < n:
            return k
