"""Shared helpers for the tests (parity metrics of the reference)."""
import numpy as np


def rel_l1(a, b, area):
    """Relative L1 error per column, MomentSolver::CalculateError
    (momentsolver.cpp:687-749): sum |a-b| area / sum |b| area."""
    a = np.asarray(a); b = np.asarray(b); w = np.asarray(area)[:, None]
    num = (np.abs(a - b) * w).sum(0)
    den = (np.abs(b) * w).sum(0)
    return num / np.where(den == 0, 1.0, den)
