"""Seeded synthetic workloads for the benchmark and the tests (splitmix64 streams).

The reference publishes no benchmark data set; every workload is generated
here from a fixed seed per configuration (seed = 0xC0DA0000 + index).
"""
from __future__ import annotations

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014); one seed per workload."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next_u64(self, n: int) -> np.ndarray:
        # vectorised: state_k = seed + k * gamma
        gamma = np.uint64(0x9E3779B97F4A7C15)
        k = np.arange(1, n + 1, dtype=np.uint64)
        with np.errstate(over="ignore"):
            z = np.uint64(self.state) + k * gamma
            self.state = int((np.uint64(self.state) + np.uint64(n) * gamma)) & MASK64
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
        return z

    def residues(self, n: int, p: int) -> np.ndarray:
        """n uniform residues in [0, p) by rejection on the top 32 bits (no % bias)."""
        out = np.empty(0, dtype=np.uint32)
        bits = int(p - 1).bit_length()
        while len(out) < n:
            z = self.next_u64(max(2 * (n - len(out)), 64)) >> np.uint64(64 - bits)
            out = np.concatenate([out, z[z < p].astype(np.uint32)])
        return out[:n]

    def int64_in(self, n: int, bound: int) -> np.ndarray:
        """n uniform integers in [-bound, bound] by rejection."""
        span = 2 * bound + 1
        bits = span.bit_length()
        out = np.empty(0, dtype=np.int64)
        while len(out) < n:
            z = self.next_u64(max(2 * (n - len(out)), 64)) >> np.uint64(64 - bits)
            z = z[z < np.uint64(span)]
            out = np.concatenate([out, z.astype(np.int64) - bound])
        return out[:n]

    def log_uniform_int(self, n: int, lo: int, hi: int) -> np.ndarray:
        u = (self.next_u64(n) >> np.uint64(11)).astype(np.float64) / float(1 << 53)
        return np.floor(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64)

    def uniform01(self, n: int) -> np.ndarray:
        return (self.next_u64(n) >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def seed_for(config_index: int) -> int:
    return 0xC0DA0000 + config_index
