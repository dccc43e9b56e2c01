"""Host-side logic of the warm-start surrogate on the CPU, with torch's conv3d standing in for the tensor-core
kernels: network shapes, the training loop, the adjoint-weight identity the data gradient relies on, and the
mapping between solver fields and the network's channels-last targets."""
import pytest
import numpy as np
import torch
import torch.nn.functional as F

from xadvcool_b200 import surrogate as S
from xadvcool_b200.designs import gyroid_design


def test_forward_shapes_cpu():
    m = S.Surrogate("cpu", seed=0)
    x = torch.randn(2, 8, 16, 24, 16).to(S.BF16)
    y = m.forward(x, S.torch_conv3d)
    assert y.shape == (2, 8, 16, 24, 16) and y.dtype == torch.float32
    assert torch.isfinite(y).all()
    # padded output channels stay exactly zero (zero weights and bias)
    assert (y[..., S.OUT_FIELDS:] == 0).all()


def test_training_loop_reduces_loss_cpu():
    torch.manual_seed(0)
    m = S.Surrogate("cpu", seed=1)
    x = torch.zeros(1, 8, 16, 24, 16)
    x[..., 0] = (torch.rand(1, 8, 16, 24) > 0.4).float()
    x[..., 1] = torch.rand(1, 8, 16, 24)
    x = x.to(S.BF16)
    y = torch.zeros(1, 8, 16, 24, S.OUT_FIELDS)
    y[..., 0] = x[..., 0].float() * (1 + x[..., 1].float())
    y[..., 4] = x[..., 1].float() ** 2
    hist = S.train(m, [(x, y)], epochs=40, batch=1, lr=3e-3, conv=S.torch_conv3d)
    assert np.isfinite(hist).all()
    assert hist[-1] < 0.3 * hist[0], hist


def test_adjoint_weights_give_data_gradient():
    """conv(dy, adjoint(w)) is the gradient of <conv(x, w), dy> with respect to x (zero padding)."""
    g = torch.Generator().manual_seed(2)
    x = torch.randn(1, 4, 5, 6, 16, generator=g).to(S.BF16).float().requires_grad_(True)
    w = torch.randn(27, 32, 16, generator=g).to(S.BF16).float()
    dy = torch.randn(1, 4, 5, 6, 32, generator=g).to(S.BF16)
    y = S.torch_conv3d(x, w, None, 3, True)
    y.backward(dy.float())
    dx = S.torch_conv3d(dy, S.adjoint_weights(w.to(S.BF16)).float(), None, 3, True)
    torch.testing.assert_close(dx, x.grad, rtol=1e-5, atol=1e-4)


def test_targets_round_trip():
    mask, hs, u_in, _ = gyroid_design(3, nx=48, ny=32, nz=16, buf=4)
    nx, ny, nz = mask.shape
    g = torch.Generator().manual_seed(3)
    rho = 1 + 0.01 * torch.randn(nx, ny, nz, generator=g)
    u = 0.03 * torch.randn(nx, ny, nz, 3, generator=g)
    T = 25 + torch.rand(nx, ny, nz, generator=g)
    solid = torch.from_numpy(mask == 1)
    inlet = torch.from_numpy(mask == 2)
    assert inlet.any()
    rho[solid], u[solid] = 1.0, 0.0
    tg = S.targets(rho, u, T, u_in, 0.1)
    assert tg.shape == (1, nz, ny, S.NXP, S.OUT_FIELDS)
    r2, u2, T2 = S.fields_from_prediction(tg, mask.shape, u_in, 0.1, mask)
    # inlet cells start exactly as a cold start does (their density is never re-derived from neighbours)
    assert (r2[inlet] == 1.0).all() and (u2[inlet] == 0.0).all() and (T2[inlet] == 25.0).all()
    rho[inlet], u[inlet], T[inlet] = 1.0, 0.0, 25.0
    torch.testing.assert_close(r2, rho, rtol=0, atol=1e-6)
    torch.testing.assert_close(u2, u, rtol=0, atol=1e-7)
    torch.testing.assert_close(T2, T, rtol=0, atol=1e-5)


def test_features_layout():
    mask, hs, u_in, _ = gyroid_design(4, nx=48, ny=32, nz=16, buf=4)
    x = S.features(mask, hs, u_in, device="cpu")
    assert x.shape == (1, 16, 32, S.NXP, 16) and x.dtype == S.BF16
    fl = x[0, ..., 0].float()
    # fluid indicator transposed to [z][y][x]; padding in x is solid (0)
    assert torch.equal(fl[:, :, :48], torch.from_numpy((mask != 1).transpose(2, 1, 0).astype(np.float32)))
    assert (fl[:, :, 48:] == 0).all()
    assert float(x[0, ..., 1].max()) == 1.0
    assert torch.allclose(x[0, ..., 2].float(), torch.tensor(20 * u_in).to(S.BF16).float())
    assert (x[0, ..., 3:] == 0).all()


def test_trained_weights_load_and_run_cpu():
    """The committed weights load and give finite outputs (the network is fully convolutional: any volume whose
    sides divide by 8 runs; a small one keeps this quick on the CPU)."""
    m = S.load_pretrained("cpu")
    assert m.norm is not None
    x = torch.zeros(1, 8, 16, 24, 16)
    x[..., 0] = 1.0
    x[0, 0, :, :, 1] = 1.0
    x[..., 2] = 0.6
    y = m.forward(x.to(S.BF16), S.torch_conv3d)
    assert y.shape == (1, 8, 16, 24, 16) and torch.isfinite(y).all()


def test_comparison_against_a_tight_solve():
    """warmstart._vs: relative delta_P / R_th differences over the designs converged in both batches, and the
    count within 0.5% on both."""
    from xadvcool_b200 import warmstart as W
    ref = {"scalars": [{"delta_P": 1.0, "R_th": 2.0}, {"delta_P": 1.0, "R_th": 2.0}, {"delta_P": 1.0, "R_th": 2.0}]}
    a = {"scalars": [{"delta_P": 1.001, "R_th": 2.002}, {"delta_P": 1.0, "R_th": 2.1}, {"delta_P": 5.0, "R_th": 9.0}]}
    r = W._vs(a, ref, [True, True, False], [True, True, True])
    assert r["compared"] == 2
    assert abs(r["dP_rel_max"] - 1e-3) < 1e-12
    assert abs(r["Rth_rel_max"] - 0.05) < 1e-12
    assert r["within_half_percent"] == 1
    assert W._vs(a, ref, [False] * 3, [True] * 3)["compared"] == 0


def test_convolution_kernels_refuse_host_tensors():
    """Host tensors are refused before any pointer reaches the library."""
    import pytest
    x = torch.zeros((1, 2, 2, 2, 16), dtype=torch.bfloat16)
    w = torch.zeros((27, 16, 16), dtype=torch.bfloat16)
    with pytest.raises(ValueError, match="CUDA tensor"):
        S.conv_forward(x, w, None, 3)
    with pytest.raises(ValueError, match="CUDA tensor"):
        S.conv_weight_grad(x, x, 3, False)


def test_compare_batched_reports_every_design(monkeypatch):
    """warmstart.compare_batched with the solves replaced by fakes: one row per design that passes the guard, in
    seed order, with None where either solve did not converge; the guard-tripping designs are skipped when asked."""
    from xadvcool_b200 import warmstart as W

    def fake_batched(ds, model, *, max_steps, tol, warm_min_steps):
        n = len(ds)
        warm = model is not None
        ok = [not (warm and j == 1) for j in range(n)]  # the second design's warm solve does not converge
        scal = [{"delta_P": 1.0 + j, "R_th": (2.0 if not warm else 2.02) + j * (tol < 1e-7)} for j in range(n)]
        steps = [(1000 if warm else 9000) + 100 * j for j in range(n)]
        return {"wall_s": float(sum(steps)), "designs": n, "converged": sum(ok), "s_per_converged_design": 1.0,
                "diverged": 0, "steps": steps, "ok": ok, "scalars": scal}

    monkeypatch.setattr(W, "_batched", fake_batched)
    monkeypatch.setattr(W, "screen", lambda seeds: ([s for s in seeds if s % 3], [s for s in seeds if not s % 3]))
    monkeypatch.setattr(W, "design", lambda s: (None, None, None, None))
    r = W.compare_batched(object(), [1, 2, 3, 4, 5], tight_tol=1e-8, solve_cold_tripped=False)
    rows = r["per_design"]
    assert [x["seed"] for x in rows] == [1, 2, 4, 5] and r["screened_out"] == 1
    assert rows[1]["Rth_warm_vs_cold"] is None and rows[1]["Rth_warm_vs_tight"] is None
    assert rows[0]["Rth_warm_vs_cold"] == pytest.approx(0.01) and rows[0]["cold_steps"] == 9000
    assert "warm_cold_tripped" not in r and r["compared"] == 3
