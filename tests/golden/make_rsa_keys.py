"""Generates tests/golden/rsa2048_keys.json: seeded RSA-2048 keys for the RSA AIR tests.

The keys are ordinary 2048-bit RSA keys (e = 65537, two 1024-bit primes with the
top two bits set) drawn from Python's seeded Mersenne Twister with a
Miller-Rabin test. They are test data for the library's own tests; nothing of
the reference is involved.

    python tests/golden/make_rsa_keys.py
"""
import json
import os
import random

E = 65537
SMALL_PRIMES = [p for p in range(3, 2000) if all(p % q for q in range(2, int(p ** 0.5) + 1))]


def probable_prime(n: int, rng: random.Random, rounds: int = 40) -> bool:
    if any(n % p == 0 for p in SMALL_PRIMES):
        return n in SMALL_PRIMES
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for _ in range(rounds):
        a = rng.randrange(2, n - 2)
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = pow(x, 2, n)
            if x == n - 1:
                break
        else:
            return False
    return True


def prime(bits: int, rng: random.Random) -> int:
    while True:
        c = rng.getrandbits(bits) | (3 << (bits - 2)) | 1
        if (c - 1) % E and probable_prime(c, rng):
            return c


def keypair(rng: random.Random):
    while True:
        p, q = prime(1024, rng), prime(1024, rng)
        n = p * q
        if p != q and n.bit_length() == 2048:
            return n, pow(E, -1, (p - 1) * (q - 1))


def main():
    rng = random.Random(0x5EED_2048)
    keys = [keypair(rng) for _ in range(4)]
    out = {"e": E, "keys": [{"n": format(n, "x"), "d": format(d, "x")} for n, d in keys]}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rsa2048_keys.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
