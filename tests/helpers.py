"""Shared helpers for the parity tests (comparisons of gauge-invariant quantities)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name="reference_kats.json"):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def cm(pairs, shape):
    """Column-major complex matrix from (re, im) pairs."""
    return np.array([complex(a, b) for a, b in pairs]).reshape(shape, order="F")


def logov_close(a, b, rtol):
    """Log-overlaps agree: real parts to rtol (relative to max(1,|.|)), phases mod 2pi."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.maximum(1.0, np.abs(b.real))
    re = np.abs(a.real - b.real) / scale
    ph = np.abs(np.exp(1j * a.imag) - np.exp(1j * b.imag))
    return float(max(re.max(initial=0.0), ph.max(initial=0.0)))


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(1e-300, np.abs(b).max()))


def divisors(n):
    """getDivisors (common/erroranalysisHao): the divisors of n in increasing order."""
    return [d for d in range(1, n + 1) if n % d == 0]


def num_den_block_analysis(num, den, min_blocks=10):
    """NumDenErrorAnalysis (afqmc/utilities/manipulateMCData/bin/NumDenErrorAnalysis.cpp:36-62)
    with getMeanError (common/erroranalysisHao/include/serialErrorAnalysis.h:18-47):
    for each block size b dividing the sample count, the per-block ratios
    sum(num)/sum(den), their mean and the error sqrt(var/(nb-1)).  Returns
    (ratio of the totals, the largest error over block sizes that leave at
    least min_blocks blocks, the per-block-size table)."""
    num = np.asarray(num)
    den = np.asarray(den)
    n = len(num)
    table = []
    for b in divisors(n):
        nb = n // b
        r = num.reshape(nb, b).sum(1) / den.reshape(nb, b).sum(1)
        mean = r.mean()
        err = np.sqrt(np.mean(np.abs(r - mean) ** 2) / (nb - 1)) if nb > 1 else 0.0
        table.append((b, mean, err))
    errs = [e for b, _, e in table if n // b >= min_blocks]
    return num.sum() / den.sum(), max(errs), table
