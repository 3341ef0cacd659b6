"""Thread-block shape enumeration of the reference's exhaustive sweep.

Restates cuda/primes.cpp:4-87 (same factor order, so a sweep visits shapes in the reference's
order): every ordered factorisation of ``warps * warpSize`` into (x, y) or (x, y, z).
"""

from __future__ import annotations


def prime_factorization(number: int) -> list:
    """[(1, 1), (p, multiplicity), ...]; the leading (1, 1) is part of the reference's contract."""
    primes = [(1, 1)]
    i = 2
    while i * i <= number:
        count = 0
        while number % i == 0:
            number //= i
            count += 1
        if count:
            primes.append((i, count))
        i += 1
    if number != 1:
        primes.append((number, 1))
    return primes


def prime_combinations(number: int) -> list:
    """All divisors of ``number`` in the reference's generation order."""
    singles = []
    for prime, count in prime_factorization(number):
        powers = []
        f = 1
        for _ in range(count):
            f *= prime
            powers.append(f)
        if prime != 1:
            powers.insert(0, 1)
        singles.append(powers)
    out = singles[0]
    for other in singles[1:]:
        out = [f * o for o in other for f in out]
    return out


def prime_combinations_2d(number: int) -> list:
    return [(f, number // f) for f in prime_combinations(number)]


def prime_combinations_3d(number: int) -> list:
    out = []
    for f1 in prime_combinations(number):
        for a, b in prime_combinations_2d(number // f1):
            out.append((f1, a, b))
    return out


def block_shapes(dimension: int, max_threads_per_block: int, warp_size: int = 32,
                 max_threads=(1024, 1024, 64)) -> list:
    """Shapes visited by Benchmark2D/Benchmark3D (cuda/benchmark.cpp:223-251,287-318)."""
    shapes = []
    for warps in range(1, max_threads_per_block // warp_size + 1):
        n = warps * warp_size
        if dimension == 2:
            for x, y in prime_combinations_2d(n):
                if x > max_threads[0] or y > max_threads[1]:
                    continue
                shapes.append((x, y, 1))
        else:
            for x, y, z in prime_combinations_3d(n):
                if x > max_threads[0] or y > max_threads[1] or z > max_threads[2]:
                    continue
                shapes.append((x, y, z))
    return shapes
