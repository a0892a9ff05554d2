"""``oceansar/utils/misc.py`` helpers used by the raw generator."""
import numpy as np


def _largest_prime(n):
    best, p = 1, 2
    while p * p <= n:
        while n % p == 0:
            best, n = p, n // p
        p += 1 if p == 2 else 2
    return max(best, n) if n > 1 else best


def optimize_fftsize(values, max_prime=2):
    """Good FFT sizes (``misc.py:60-83``): next power of two for ``max_prime == 2``, else
    the next integer whose largest prime factor is <= ``max_prime``."""
    scalar = np.isscalar(values)
    vals = np.atleast_1d(np.array(values, dtype=int))
    if max_prime == 2:
        good = (2 ** np.ceil(np.log2(vals))).astype(int)
    else:
        good = []
        for v in vals:
            b = int(v)
            while _largest_prime(b) > max_prime:
                b += 1
            good.append(b)
        good = np.array(good, dtype=int)
    return good[0] if (scalar or good.size == 1) else good


def db(a, linear=False):
    return 20 * np.log10(np.abs(a)) if linear else 10 * np.log10(np.abs(a))


def db2lin(a, amplitude=False):
    return 10 ** (a / 20) if amplitude else 10 ** (a / 10)
