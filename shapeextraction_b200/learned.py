"""Learned search-radius proposal: training and use.

The model (a 32 -> 64 -> 64 -> 1 MLP, BF16 weights and activations, FP32
accumulation) predicts y = log2(r_k^2 / range^2) for every tree point from
occupancy features of the built tree, where r_k is the distance to the point's
k-th neighbour and range the cloud's extent. Training targets are the exact
k-th-neighbour distances of the plain search on a held-out cloud; training runs
on the GPU through the C ABI (se_mlp_train: the library's forward, backward and
Adam kernels). A log-margin, set from a high quantile of the training
residuals, turns predictions into upper bounds; the search starts from that
bound and re-searches, without it, any query it underestimates, so kNN stays
exact whatever the model predicts.
"""
from __future__ import annotations

import numpy as np

from ._native import Context

B3 = 6336  # index of the output bias in the flat parameter vector


def radius_targets(ctx: Context, k: int, start: int = 0, count: int | None = None) -> np.ndarray:
    """log2(r_k^2 / range^2) of tree points [start, start+count), from the exact search."""
    info = ctx.info()
    rng = float(info["max_coord"]) - float(info["min_coord"])
    _, d2 = ctx.knn_self(k, start, count, with_d2=True)
    r2 = np.maximum(d2[:, k - 1].astype(np.float64), 1e-30)
    return (np.log2(r2) - 2.0 * np.log2(rng)).astype(np.float32)


def _sample(ctx: Context, k: int, max_rows: int, rng) -> tuple[np.ndarray, np.ndarray]:
    """Features and targets of all points, or of 64 random Morton-contiguous
    chunks (spread over the cloud) when it has more than max_rows points."""
    u = ctx.info()["n_points"]
    if u <= max_rows:
        return ctx.features(), radius_targets(ctx, k)
    chunk = max(1, max_rows // 64)
    starts = np.sort(rng.choice(u // chunk, size=64, replace=False)) * chunk
    X = np.concatenate([ctx.features(int(s), chunk) for s in starts])
    y = np.concatenate([radius_targets(ctx, k, int(s), chunk) for s in starts])
    return X, y


def train_radius_model(ctx: Context, k: int, steps: int = 1500, batch: int = 8192, lr: float = 2e-3, seed: int = 0,
                       quantile: float = 0.995, max_rows: int = 1_000_000, pinball: float = 0.0,
                       pinball_steps: int = 500) -> dict:
    """Train the context's model on its own built cloud (the held-out cloud)
    and calibrate the margin at the `quantile` of the training residuals.
    A warp searches again whenever one of its 32 lanes misses, so misses cost
    far more than a slightly looser bound: 0.995 measured best on surface,
    mixture and precision-mix clouds (0.99 and 0.999 were 1-4% slower).
    With pinball in (0, 1) the squared-error training is followed by
    pinball_steps steps of the pinball loss of that quantile, so that the
    network predicts a per-point upper bound and the global margin covers
    only the rest. Returns the losses and the calibration."""
    rng = np.random.default_rng(seed)
    X, y = _sample(ctx, k, max_rows, rng)
    perm = rng.permutation(y.size)
    Xs, ys = np.ascontiguousarray(X[perm]), np.ascontiguousarray(y[perm])
    ctx.mlp_init(seed)
    p = ctx.mlp_params()
    p[B3] = float(ys.mean())
    ctx.mlp_params(p)
    ctx.mlp_set_loss(0.0)
    losses = ctx.mlp_train(Xs, ys, steps, batch, lr)
    if pinball > 0.0 and pinball_steps > 0:
        ctx.mlp_set_loss(pinball)
        losses = np.concatenate([losses, ctx.mlp_train(Xs, ys, pinball_steps, batch, lr * 0.5)])
        ctx.mlp_set_loss(0.0)
    # calibrate with the training forward over the same rows; the tensor-core
    # path that queries use differs from it by far less than the 0.02 added
    yhat = np.concatenate([ctx.mlp_forward(Xs[i:i + 1_000_000]) for i in range(0, ys.size, 1_000_000)])
    res = ys.astype(np.float64) - yhat
    margin = float(np.quantile(res, quantile)) + 0.02
    ctx.mlp_set_margin(margin)
    return {"losses": losses, "margin": margin, "quantile": quantile, "rows": int(ys.size),
            "residual_std": float(res.std()), "target_mean": float(y.mean()), "pinball": pinball}


def transfer(src: Context, dst: Context, margin: float) -> None:
    """Copy a trained model (parameters and margin) into another context."""
    dst.mlp_params(src.mlp_params())
    dst.mlp_set_margin(margin)
