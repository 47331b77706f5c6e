"""FP64 restatement of the VNLB group filter.  TEST INFRASTRUCTURE ONLY.

The reference computes the filter in FP32 (src/core/core.cpp
filter_vnlb_samples, :638-781).  This module computes the same mathematics in
float64 with numpy, so that tests can state how far each GPU form is from the
exact result: the plain form (the reference's FP32 arithmetic) and the chosen
forms (TF32 tensor-core Gram with FP32 accumulation, FP64 Jacobi angles).
Covered: coupled groups on the dual-PCA model (dimension >= 64, model rows
below the dimension), the configuration of the bench workload.

Steps, each following the reference function named:
  * flat-area test (Final): is_flat_samples_group / samples_channel_variance
    (core.cpp:533-576), mean over channels of the unbiased variance;
  * means of the first B rows, centring (filter_vnlb_samples, core.cpp:638-697;
    linalg compute_mean / center_rows);
  * dual Gram X X^T / B of the centred model rows (compute_gram_centered,
    src/linalg/linalg.cpp:326-354);
  * top-r eigenpairs, descending (topk_symmetric_eigen_jacobi,
    linalg.cpp:447-519; here numpy's symmetric eigensolver in float64);
  * dual -> primal basis u_i = X^T v_i / sqrt(lambda_i), zero when lambda_i is at
    most 128 FLT_EPSILON, then normalised (map_dual_eigenvectors_to_basis,
    linalg.cpp:552-595);
  * Wiener coefficients (compute_filter_coefficients, core.cpp:616-636) and
    the projection plus centre (project_bayes_estimate, core.cpp:578-614).
"""
from __future__ import annotations

import numpy as np

FLT_EPSILON = float(np.finfo(np.float32).eps)


def group_rows(clip: np.ndarray, rows, patch_size: int, patch_time: int) -> np.ndarray:
    """The coupled sample rows [S][D] of matches (x, y, frame) in float64,
    columns ordered (channel, t, py, px) as the reference gathers them
    (gather_*, core.cpp:1364-1585)."""
    frames, channels, h, w = clip.shape
    out = np.empty((len(rows), channels * patch_time * patch_size * patch_size), np.float64)
    for i, (x, y, f) in enumerate(rows):
        block = clip[f:f + patch_time, :, y:y + patch_size, x:x + patch_size]  # [t][c][py][px]
        out[i] = np.transpose(block, (1, 0, 2, 3)).reshape(-1)
    return out


def filter_group(stage: int, params, noisy_rows: np.ndarray, basic_rows: np.ndarray | None, channels: int,
                 patch_dim: int) -> np.ndarray:
    """Filtered rows [S][D] (float64) of one coupled dual-PCA group."""
    S, D = noisy_rows.shape
    cap = model_cap(params.similar, params.model_cap_factor)
    B = min(S, cap)
    rank = min(params.rank, D)
    beta, sigma = float(np.float32(params.beta)), float(np.float32(params.sigma))
    sigma2 = beta * sigma * sigma
    if stage == 1:
        sb = float(np.float32(params.sigma_basic))
        sigma_b2 = beta * sb * sb
    else:
        sigma_b2 = sigma2
    mean_n = noisy_rows[:B].mean(axis=0)
    if stage == 1:
        mean_b = basic_rows[:B].mean(axis=0)
        model = basic_rows[:B] - mean_b
        flat = bool(params.flat_areas) and channel_variance(noisy_rows, channels, patch_dim) < (
            sigma * sigma * float(np.float32(params.gamma)))
        center = mean_b if flat else mean_n
        centred = noisy_rows - center
    else:
        model = noisy_rows[:B] - mean_n
        center = mean_n
        centred = noisy_rows - mean_n
    if rank == 0:
        return np.tile(center, (S, 1))
    gram = model @ model.T / B
    lam, vec = np.linalg.eigh(gram)
    order = np.argsort(lam)[::-1][:rank]
    lam, vec = lam[order], vec[:, order]
    basis = np.zeros((rank, D))
    for i in range(rank):
        if lam[i] > 128.0 * FLT_EPSILON:
            u = model.T @ vec[:, i] / np.sqrt(lam[i])
            n = np.sqrt(u @ u)
            basis[i] = u / n if n > 128.0 * FLT_EPSILON else 0.0
    variance = lam - np.minimum(lam, sigma_b2) if sigma_b2 > 0.0 else lam.copy()
    threshold = float(np.float32(params.variance_threshold)) * sigma2
    coef = np.where(variance > threshold, 1.0 / (1.0 + sigma2 / np.maximum(variance, 1e-300)), 0.0)
    proj = centred @ basis.T  # [S][rank]
    return center + (proj * coef) @ basis


def channel_variance(rows: np.ndarray, channels: int, patch_dim: int) -> float:
    """samples_channel_variance (core.cpp:533-559) in float64."""
    total = 0.0
    for c in range(channels):
        v = rows[:, c * patch_dim:(c + 1) * patch_dim].reshape(-1)
        if v.size <= 1:
            return 0.0
        total += v.var(ddof=1)
    return total / channels


def model_cap(similar: int, factor: float) -> int:
    """model_similar_cap (core.cpp:159-172)."""
    if factor == 0.0:
        return 1 << 30
    return max(similar, int(np.ceil(np.float32(similar) * np.float32(factor))))
