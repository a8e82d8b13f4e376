"""Shared helpers of the test-suite (error metrics, golden loading, workloads)."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name))


def row_rel_err(got: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Per-row |got - ref| / |ref| (vector norm over the 3 components)."""
    num = np.linalg.norm(got - ref, axis=1)
    den = np.linalg.norm(ref, axis=1)
    return num / np.maximum(den, 1e-300)


def lists_equal(nnb_a, list_a, nnb_b, list_b) -> bool:
    if not np.array_equal(np.asarray(nnb_a), np.asarray(nnb_b)):
        return False
    for r in range(len(nnb_a)):
        k = int(nnb_a[r])
        if not np.array_equal(list_a[r, :k], list_b[r, :k]):
            return False
    return True


def first_list_mismatch(nnb_a, list_a, nnb_b, list_b):
    for r in range(len(nnb_a)):
        ka, kb = int(nnb_a[r]), int(nnb_b[r])
        if ka != kb or not np.array_equal(list_a[r, :ka], list_b[r, :kb]):
            return r, list_a[r, :ka], list_b[r, :kb]
    return None
