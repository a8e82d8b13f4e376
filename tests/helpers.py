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


ACC_TOL = 1e-6
JERK_TOL = 1e-5
IRR_TOL = 1e-12


def check_force(res, ref, tag, scale, acc_tol=ACC_TOL, jerk_tol=JERK_TOL):
    """Lists exact; forces within the bar of tests/test_regforce_gpu.py:
    per target |da| <= acc_tol |a| + 0.1 acc_tol A (A = sum of the magnitudes of
    the regular acc terms, ``scale[0]``), the same for jerk with ``scale[1]``;
    norm-wise over calls of more than 16 rows; the FP64 irregular part to
    IRR_TOL.  Returns the measured figures, including how many rows the first
    (relative) term alone would have failed -- the rows that needed the FP32
    summation floor."""
    mm = first_list_mismatch(res.nnb, res.list, ref["nnb"], ref["list"])
    assert mm is None, f"{tag}: list mismatch at row {mm}"
    da = np.linalg.norm(res.acc_reg - ref["acc_reg"], axis=1)
    dj = np.linalg.norm(res.jerk_reg - ref["jerk_reg"], axis=1)
    na = np.linalg.norm(ref["acc_reg"], axis=1)
    nj = np.linalg.norm(ref["jerk_reg"], axis=1)
    ea = da / np.maximum(acc_tol * na + 0.1 * acc_tol * scale[0], 1e-300)
    ej = dj / np.maximum(jerk_tol * nj + 0.1 * jerk_tol * scale[1], 1e-300)
    rel_a = row_rel_err(res.acc_reg, ref["acc_reg"])
    rel_j = row_rel_err(res.jerk_reg, ref["jerk_reg"])
    norm_a = np.linalg.norm(da) / max(np.linalg.norm(na), 1e-300)
    norm_j = np.linalg.norm(dj) / max(np.linalg.norm(nj), 1e-300)
    floor_a = int(np.count_nonzero(da > acc_tol * na))
    floor_j = int(np.count_nonzero(dj > jerk_tol * nj))
    print(f"{tag}: rows {na.size} | rel acc max {rel_a.max():.2e} med {np.median(rel_a):.2e} "
          f"norm {norm_a:.2e} | jerk max {rel_j.max():.2e} med {np.median(rel_j):.2e} norm {norm_j:.2e} | "
          f"bound use acc {ea.max():.2f} jerk {ej.max():.2f} | rows needing the floor: acc {floor_a} "
          f"jerk {floor_j} | plan {getattr(res, 'plan', None)}")
    assert ea.max() <= 1.0, f"{tag}: acc error {ea.max():.2f} x the bound"
    assert ej.max() <= 1.0, f"{tag}: jerk error {ej.max():.2f} x the bound"
    if na.size > 16:
        assert norm_a <= acc_tol and norm_j <= jerk_tol, f"{tag}: norm-wise {norm_a:.2e} {norm_j:.2e}"
    has = ref["nnb"] > 0
    if has.any():
        ei = row_rel_err(res.acc_irr[has], ref["acc_irr"][has])
        eij = row_rel_err(res.jerk_irr[has], ref["jerk_irr"][has])
        assert ei.max() <= IRR_TOL and eij.max() <= IRR_TOL, f"{tag}: irregular {ei.max()} {eij.max()}"
    return dict(rows=int(na.size), acc_max=float(rel_a.max()), acc_med=float(np.median(rel_a)),
                jerk_max=float(rel_j.max()), jerk_med=float(np.median(rel_j)), norm_acc=float(norm_a),
                norm_jerk=float(norm_j), bound_use_acc=float(ea.max()), bound_use_jerk=float(ej.max()),
                floor_rows_acc=floor_a, floor_rows_jerk=floor_j)
