"""Synthetic ragged workloads (shapes only; no data).

* ``ragged_mix``: polynomials with logN, limb count and operation drawn from
  a seed, each with its own modulus chain: ``limbs`` consecutive primes
  q == 1 (mod 2N) above 2^29.5 (30-bit) or 2^30.5 (31-bit), starting at a
  seeded offset into the first ``pool`` such primes.  Distinct polynomials
  therefore have distinct but overlapping chains, as RNS levels do.

Used by the batch / serving tests and by bench.py.
"""
from __future__ import annotations

import functools
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import OP_FORWARD, OP_INVERSE, OP_MULTIPLY, find_moduli

BITS_START = {30: int(2 ** 29.5), 31: int(2 ** 30.5)}


@dataclass
class MixJob:
    op: int
    logN: int
    moduli: List[Tuple[int, int]]

    @property
    def limbs(self) -> int:
        return len(self.moduli)

    @property
    def words(self) -> int:
        return self.limbs << self.logN


@functools.lru_cache(maxsize=None)
def prime_pool(logN: int, bits: int, pool: int) -> Tuple[Tuple[int, int], ...]:
    return tuple((m.qi, m.primitive_root) for m in find_moduli(logN, pool, BITS_START[bits]))


def ragged_mix(seed: int = 1234, count: int = 256, logn: Sequence[int] = (12, 16),
               limbs: Tuple[int, int] = (1, 48), bits: Sequence[int] = (30,),
               ops: Sequence[Tuple[int, float]] = ((OP_FORWARD, 1.0),),
               pool: int = 96) -> List[MixJob]:
    """`logn`: the logN values drawn uniformly; `limbs`: inclusive range;
    `bits`: modulus widths drawn uniformly; `ops`: (op, weight) pairs."""
    rng = np.random.default_rng(seed)
    opv = np.array([o for o, _ in ops])
    opw = np.array([w for _, w in ops], dtype=float)
    opw /= opw.sum()
    out = []
    for _ in range(count):
        lg = int(rng.choice(np.asarray(logn)))
        L = int(rng.integers(limbs[0], limbs[1] + 1))
        b = int(rng.choice(np.asarray(bits)))
        P = prime_pool(lg, b, max(pool, L))
        off = int(rng.integers(0, len(P) - L + 1))
        out.append(MixJob(int(rng.choice(opv, p=opw)), lg, list(P[off:off + L])))
    return out


def uniform_device(torch, job: MixJob, gen) -> "torch.Tensor":
    """A (limbs, N) int32 CUDA tensor, limb l uniform in [0, q_l)."""
    q = torch.tensor([m[0] for m in job.moduli], dtype=torch.int64, device="cuda")
    x = torch.randint(0, 1 << 62, (job.limbs, 1 << job.logN), dtype=torch.int64, device="cuda",
                      generator=gen)
    return (x % q[:, None]).to(torch.int32)
