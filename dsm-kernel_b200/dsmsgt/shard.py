"""Frequency ownership across ranks (one process per GPU).

Frequencies are independent units with no exchange step, so ranks share no
data: each rank computes the frequencies it owns and writes their catalogue
records.  Ownership follows the reference's zig-zag rule
(src/SGTpsv/SGTpsv-MPI.f90:550, src/SGTsh/SGTsh-MPI.f90:403): frequency
i != 0 belongs to rank p of n when (imax - p - i) or (imax + p + 1 - i) is a
multiple of 2n, which pairs high and low frequencies on every rank and so
balances the cost (the angular-order cutoff grows with frequency)."""
from __future__ import annotations


def owns(i: int, imax: int, rank: int, nproc: int) -> bool:
    if i == 0:
        return False
    return (imax - rank - i) % (2 * nproc) == 0 or (imax + rank + 1 - i) % (2 * nproc) == 0


def owned_freqs(imin: int, imax: int, rank: int, nproc: int) -> list[int]:
    return [i for i in range(imin, imax + 1) if owns(i, imax, rank, nproc)]
