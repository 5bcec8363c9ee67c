"""Seeded Poisson sampling as the reference's simulator draws it (oracle restatement, test
infrastructure only).

physwkim/ptyrs `base/sim.rs:143-175` (`poisson`) draws each pixel's count from
`rand_distr::Poisson` (rand_distr 0.4.3) with one `rand_chacha::ChaCha8Rng` (rand_chacha
0.3.1) stream seeded by `SeedableRng::seed_from_u64` (rand_core 0.6). None of those crates is
vendored under the reference, so their published algorithms are restated here:

- `seed_from_u64`: the 32-byte seed filled with PCG32 outputs (multiplier 6364136223846793005,
  increment 11634580027462260723, state advanced before each output, XSH-RR output), four
  little-endian bytes at a time;
- ChaCha with 8 rounds (Bernstein): the "expand 32-byte k" constants, the seed as the key, a
  64-bit block counter from 0 in words 12-13 and stream 0 in words 14-15; the generator hands
  out the 32-bit words of blocks in counter order, `next_u64` as two words (low first) across
  its 64-word buffer as `rand_core::block::BlockRng` does;
- `Standard` f64: the top 53 bits of `next_u64` times 2^-53;
- `Poisson`: Knuth's product of uniforms below λ = 12, above it the rejection method of
  Numerical Recipes against a Cauchy comparison (`tan(π·u)`), with the Lanczos `log_gamma` of
  Numerical Recipes' `gammln` coefficients.

Transcendental functions go through Python's `math` (the platform libm, as Rust's f64 methods).
"""
import math

import numpy as np

_M32 = 0xFFFFFFFF
_M64 = 0xFFFFFFFFFFFFFFFF


def _rotl(v, n):
    return ((v << n) | (v >> (32 - n))) & _M32


def seed_from_u64(state):
    """rand_core 0.6 `SeedableRng::seed_from_u64` for a 32-byte seed: eight u32 key words."""
    mul, inc = 6364136223846793005, 11634580027462260723
    words = []
    for _ in range(8):
        state = (state * mul + inc) & _M64
        xorshifted = (((state >> 18) ^ state) >> 27) & _M32
        rot = state >> 59
        words.append(((xorshifted >> rot) | (xorshifted << ((32 - rot) & 31))) & _M32)
    return words


def chacha_block(key, counter, rounds=8):
    """One 16-word ChaCha block (64-bit counter, stream 0)."""
    init = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574] + list(key) + [
        counter & _M32, (counter >> 32) & _M32, 0, 0]
    x = list(init)

    def qr(a, b, c, d):
        x[a] = (x[a] + x[b]) & _M32
        x[d] = _rotl(x[d] ^ x[a], 16)
        x[c] = (x[c] + x[d]) & _M32
        x[b] = _rotl(x[b] ^ x[c], 12)
        x[a] = (x[a] + x[b]) & _M32
        x[d] = _rotl(x[d] ^ x[a], 8)
        x[c] = (x[c] + x[d]) & _M32
        x[b] = _rotl(x[b] ^ x[c], 7)

    for _ in range(rounds // 2):
        qr(0, 4, 8, 12)
        qr(1, 5, 9, 13)
        qr(2, 6, 10, 14)
        qr(3, 7, 11, 15)
        qr(0, 5, 10, 15)
        qr(1, 6, 11, 12)
        qr(2, 7, 8, 13)
        qr(3, 4, 9, 14)
    return [(a + b) & _M32 for a, b in zip(x, init)]


class ChaCha8Rng:
    """rand_chacha 0.3.1 `ChaCha8Rng::seed_from_u64(seed)`."""

    def __init__(self, seed):
        self.key = seed_from_u64(seed)
        self.counter = 0
        self.results = []
        self.index = 64

    def _generate(self):
        self.results = []
        for b in range(4):
            self.results += chacha_block(self.key, self.counter + b)
        self.counter += 4

    def next_u32(self):
        if self.index >= 64:
            self._generate()
            self.index = 0
        v = self.results[self.index]
        self.index += 1
        return v

    def next_u64(self):
        i = self.index
        if i < 63:
            self.index += 2
            return self.results[i] | (self.results[i + 1] << 32)
        if i >= 64:
            self._generate()
            self.index = 2
            return self.results[0] | (self.results[1] << 32)
        lo = self.results[63]
        self._generate()
        self.index = 1
        return lo | (self.results[0] << 32)

    def uniform(self):
        """rand 0.8 `Standard` f64 in [0, 1)."""
        return (self.next_u64() >> 11) * (1.0 / (1 << 53))


def log_gamma(x):
    """rand_distr 0.4.3 `utils::log_gamma` (Numerical Recipes `gammln`)."""
    coefficients = [76.18009172947146, -86.50532032941677, 24.01409824083091,
                    -1.231739572450155, 0.1208650973866179e-2, -0.5395239384953e-5]
    tmp = x + 5.5
    log = (x + 0.5) * math.log(tmp) - tmp
    a = 1.000000000190015
    denom = x
    for c in coefficients:
        denom = denom + 1.0
        a = a + c / denom
    return log + math.log(2.5066282746310005 * a / x)


def poisson(rng, lam):
    """rand_distr 0.4.3 `Poisson::new(lam).sample(rng)` for `lam > 0`, as f64."""
    if lam < 12.0:
        exp_lambda = math.exp(-lam)
        result = 0.0
        p = 1.0
        while p > exp_lambda:
            p = p * rng.uniform()
            result = result + 1.0
        return result - 1.0
    log_lambda = math.log(lam)
    sqrt_2lambda = math.sqrt(2.0 * lam)
    magic_val = lam * log_lambda - log_gamma(1.0 + lam)
    while True:
        while True:
            comp_dev = math.tan(math.pi * rng.uniform())
            result = sqrt_2lambda * comp_dev + lam
            if result >= 0.0:
                break
        result = math.floor(result)
        check = 0.9 * (1.0 + comp_dev * comp_dev) * math.exp(
            result * log_lambda - log_gamma(1.0 + result) - magic_val)
        if rng.uniform() <= check:
            return result


def sample_counts(intensity, seed, detector_mask=None):
    """`base::sim::poisson` (base/sim.rs:143-175): one ChaCha8 stream over the pixels in order;
    masked detector pixels (`detector_mask` `[ny, nx]`, True = masked) take no draw and store
    the mask sentinel (returned as -1); λ ≤ 0 gives 0 without a draw."""
    intensity = np.asarray(intensity, np.float64)
    shape = intensity.shape
    flat = intensity.ravel()
    plane = shape[-1] * shape[-2]
    rng = ChaCha8Rng(seed)
    out = np.empty(flat.size, np.float64)
    mask = None if detector_mask is None else np.asarray(detector_mask, bool).ravel()
    for i, lam in enumerate(flat):
        if mask is not None and mask[i % plane]:
            out[i] = -1.0
        elif lam > 0.0:
            out[i] = poisson(rng, float(lam))
        else:
            out[i] = 0.0
    return out.reshape(shape)
