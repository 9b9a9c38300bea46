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
