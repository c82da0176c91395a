"""Learned schedule cost model.

CPU: the oracle's hand-written chain rule is pinned by finite differences; the
class space, targets and regret arithmetic are checked on fixed numbers; the
committed measured dataset is well formed.
GPU: dtc_features equals the oracle's features; the MLP forward, backward
(gradients) and Adam kernels match the FP64 oracle; training is bitwise
reproducible; and on the committed dataset's held-out matrices the trained
network beats the untuned default schedule and has lower regret against the
exhaustive autotuner.
"""
import os

import numpy as np
import pytest

from oracle import costmodel_oracle as CO
from dtc_b200 import costmodel as cm

DIMS = (48, 64, 64, cm.K)


def _rand_params(dims, seed=0, scale=0.3):
    n = sum(a * b + b for a, b in zip(dims[:-1], dims[1:]))
    return np.random.default_rng(seed).standard_normal(n).astype(np.float32) * scale


def test_oracle_gradients_match_finite_differences():
    dims = (5, 7, 6, 4)
    p = _rand_params(dims, 1).astype(np.float64)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((9, 5))
    T = rng.standard_normal((9, 4))
    Mk = (rng.random((9, 4)) < 0.7).astype(np.float64)
    _, g = CO.loss_and_grads(p, dims, X, T, Mk)
    h = 1e-6
    for i in rng.choice(len(p), 25, replace=False):
        e = np.zeros_like(p)
        e[i] = h
        fd = (CO.loss_and_grads(p + e, dims, X, T, Mk)[0] -
              CO.loss_and_grads(p - e, dims, X, T, Mk)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_class_space():
    # reorder x block shape (16x8, 32x8, 16x16) x form x (window-mode waves +
    # balance-mode waves) x N-tile
    assert cm.K == 2 * 3 * 2 * (7 + 5) * 3
    assert cm.feasible(128).sum() == cm.K // 3
    # at window height 32 and at compaction width 16 the split kernels hold at
    # most 2 N-tiles per CTA
    assert cm.feasible(512).sum() == cm.K // 3 + 2 * (2 * cm.K // 9)
    d = cm.CLASSES[cm.default_class(512)]
    assert (d["H"], d["W"], d["mode"], d["waves"], d["ntile"], d["form"], d["reorder"]) == \
        (16, 8, 1, 16, 4, "split24x3", 0)
    assert {(c["H"], c["W"]) for c in cm.CLASSES} == {(16, 8), (32, 8), (16, 16)}
    assert len({cm.class_of(c["mode"], c["waves"], c["ntile"], c["form"], c["reorder"], c["H"],
                            c["W"]) for c in cm.CLASSES}) == cm.K


def test_merge_orders_slices_by_matrix_index():
    """Slices measured in separate runs merge into one dataset in matrix order,
    with the classes infeasible for each matrix's N set to NaN."""
    def part(idx):
        return dict(features=np.array([[float(i)] * 3 for i in idx]),
                    times=np.array([[float(i)] * cm.K for i in idx]),
                    meta=[dict(index=i, N=512 if i % 2 else 128,
                               split="train" if i < 4 else "test") for i in idx])
    ds = cm.merge([part([4, 5]), part([0, 1, 2]), part([3])])
    assert [m["index"] for m in ds["meta"]] == [0, 1, 2, 3, 4, 5]
    assert np.array_equal(ds["features"][:, 0], np.arange(6.0))
    for i, m in enumerate(ds["meta"]):
        f = cm.feasible(m["N"]).astype(bool)
        assert (ds["times"][i][f] == float(i)).all() and np.isnan(ds["times"][i][~f]).all()


def test_targets_and_regret():
    t = np.full((2, cm.K), np.nan, np.float32)
    t[0, :4] = [2.0, 1.0, 4.0, 1.5]
    t[1, :] = 3.0
    t[1, cm.default_class(128)] = 6.0
    y, mk = cm.targets(t)
    assert mk[0].sum() == 4 and mk[1].sum() == cm.K
    np.testing.assert_allclose(y[0, :4], np.log([2.0, 1.0, 4.0, 1.5]), rtol=1e-6)
    t[0, cm.default_class(128)] = 2.0
    ev = cm.evaluate(np.array([1, 0]), t, np.array([128, 128]))
    assert ev["regret_mean"] == pytest.approx(0.0)
    assert ev["default_regret_mean"] == pytest.approx((1.0 + 1.0) / 2)
    assert ev["speedup_vs_default_geomean"] == pytest.approx(2.0)


def test_committed_dataset_well_formed():
    if not os.path.exists(cm.DATASET_PATH):
        pytest.skip("no measured dataset committed")
    ds = cm.load_dataset()
    S = len(ds["meta"])
    assert ds["features"].shape == (S, 48) and ds["times"].shape == (S, cm.K)
    tr, N = cm.split(ds)
    assert tr.sum() > 0 and (~tr).sum() > 0
    for i in range(S):
        f = cm.feasible(int(N[i])).astype(bool)
        assert np.isfinite(ds["times"][i][f]).all() and np.isnan(ds["times"][i][~f]).all()
    assert {m["family"] for m in ds["meta"]} == set(cm.FAMILIES)


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small_uniform", "hub", "empty_windows", "banded_dense"])
def test_features_match_oracle(cuda, name):
    import torch
    from oracle import oracle as O
    from dtc_b200 import metcf
    from tests.golden import cases
    rp, col, val, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M)
    got = cm.features(torch.from_numpy(rp), torch.from_numpy(col), m, 128).cpu().numpy()
    ref = CO.features(rp, col, M, O.metcf(rp, col, M), 128)
    logs = [36, 37, 38, 39, 40, 41]
    exact = [i for i in range(48) if i not in logs]
    np.testing.assert_array_equal(got[exact], ref[exact])
    np.testing.assert_allclose(got[logs], ref[logs], rtol=1e-6)


@pytest.mark.gpu
def test_mlp_forward_backward_adam_match_oracle(cuda):
    import torch
    rng = np.random.default_rng(3)
    p = _rand_params(DIMS, 4, scale=0.2)
    net = cm.MLP(DIMS, params=p)
    B = 37
    X = rng.random((B, 48)).astype(np.float32)
    T = rng.standard_normal((B, cm.K)).astype(np.float32)
    Mk = (rng.random((B, cm.K)) < 0.5).astype(np.float32)
    H1, H2, Y = (t.cpu().numpy() for t in net.forward(X))
    rH1, rH2, rY = CO.forward(p, DIMS, X)
    np.testing.assert_allclose(Y, rY, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(H2, rH2, rtol=1e-5, atol=1e-5)
    loss, g = net.loss_and_grads(X, T, Mk)
    rl, rg = CO.loss_and_grads(p, DIMS, X, T, Mk)
    assert float(loss.item()) == pytest.approx(rl, rel=1e-5)
    g = g.cpu().numpy()
    np.testing.assert_allclose(g, rg, rtol=1e-4, atol=1e-5 * np.abs(rg).max())
    m0 = torch.zeros(net.n, device="cuda")
    v0 = torch.zeros(net.n, device="cuda")
    gd = torch.from_numpy(rg.astype(np.float32)).cuda()
    from dtc_b200._lib import call
    from dtc_b200.metcf import _ptr, _stream
    for step in (1, 2):
        call("dtc_mlp_adam", _ptr(net.params), _ptr(gd), _ptr(m0), _ptr(v0), net.n, 1e-3, 0.9,
             0.999, 1e-8, step, _stream())
    rp_, rm, rv = CO.adam(p, rg.astype(np.float32), np.zeros(net.n), np.zeros(net.n), 1e-3, 0.9,
                          0.999, 1e-8, 1)
    rp_, rm, rv = CO.adam(rp_, rg.astype(np.float32), rm, rv, 1e-3, 0.9, 0.999, 1e-8, 2)
    np.testing.assert_allclose(net.params.cpu().numpy(), rp_, rtol=1e-5, atol=1e-7)


@pytest.mark.gpu
def test_argmin_respects_feasibility(cuda):
    net = cm.MLP(DIMS, params=_rand_params(DIMS, 5))
    X = np.random.default_rng(6).random((8, 48)).astype(np.float32)
    _, _, Y = net.forward(X)
    Y = Y.cpu().numpy()
    feas = cm.feasible(128)
    ch = net.choose(X, feas)
    for r in range(8):
        ok = np.flatnonzero(feas)
        assert ch[r] == ok[np.argmin(Y[r, ok])]


@pytest.mark.gpu
def test_training_reproducible_and_descends(cuda):
    rng = np.random.default_rng(7)
    X = rng.random((64, 48)).astype(np.float32)
    T = rng.random((64, cm.K)).astype(np.float32)
    Mk = np.ones_like(T)
    a = cm.MLP(DIMS, seed=1)
    b = cm.MLP(DIMS, seed=1)
    ha = a.train(X, T, Mk, steps=200, log_every=50)
    b.train(X, T, Mk, steps=200)
    assert np.array_equal(a.params.cpu().numpy().view(np.uint32),
                          b.params.cpu().numpy().view(np.uint32))
    assert ha[-1][1] < 0.5 * ha[0][1]


@pytest.mark.gpu
def test_trained_model_beats_default_on_held_out(cuda):
    """What the network gains over the method without it, on held-out matrices."""
    if not os.path.exists(cm.DATASET_PATH):
        pytest.skip("no measured dataset committed")
    ds = cm.load_dataset()
    net, ev = cm.fit(ds, steps=2000, seed=0)
    assert ev["speedup_vs_default_geomean"] > 1.0, ev
    assert ev["regret_mean"] < ev["default_regret_mean"], ev
    assert ev["regret_median"] < 0.10, ev
    assert ev["regret_top4_mean"] <= ev["regret_mean"], ev


@pytest.mark.gpu
def test_scheduler_verifies_top_predictions(cuda):
    """Model-guided search: the plan is the fastest of the model's k cheapest
    predicted classes, timed on the caller's matrix."""
    if not os.path.exists(cm.WEIGHTS_PATH):
        pytest.skip("no trained weights committed")
    import torch
    from dtc_b200 import gen, metcf
    A = gen.zipf(20000, seed=4)
    rp, col = torch.from_numpy(A.rowptr).cuda(), torch.from_numpy(A.col).cuda()
    m = metcf.convert(rp, col, A.M, values=torch.from_numpy(A.val).cuda())
    s = cm.Scheduler()
    plain = s.plan(rp, col, m, 128)
    ver = s.plan(rp, col, m, 128, verify_top=3)
    assert plain.source == "model" and ver.source == "model+verify"
    _, _, Y = s.net.forward(cm.features(rp, col, m, 128).reshape(1, -1))
    y = Y[0].cpu().numpy()
    ok = np.flatnonzero(cm.feasible(128))
    top = set(ok[np.argsort(y[ok], kind="stable")[:3]].tolist())
    assert plain.cls in top and ver.cls in top


def test_committed_weights_beat_default_on_held_out_cpu():
    """The shipped network, evaluated by the FP64 oracle forward pass on the
    committed held-out matrices (no GPU): its choices beat the untuned default
    and stay close to the exhaustive best."""
    if not (os.path.exists(cm.DATASET_PATH) and os.path.exists(cm.WEIGHTS_PATH)):
        pytest.skip("no dataset / weights committed")
    z = np.load(cm.WEIGHTS_PATH)
    dims = tuple(int(d) for d in z["dims"])
    assert dims == DIMS
    ds = cm.load_dataset()
    tr, N = cm.split(ds)
    _, _, Y = CO.forward(z["params"], dims, ds["features"][~tr])
    choices = []
    for y, n in zip(Y, N[~tr]):
        ok = np.flatnonzero(cm.feasible(int(n)))
        choices.append(int(ok[np.argmin(y[ok])]))
    ev = cm.evaluate(np.array(choices), ds["times"][~tr], N[~tr], pred=Y, topk=8)
    # 432 classes learned from 600 matrices: the single choice is within a few
    # per cent of the exhaustive best on average, and timing the 8 cheapest
    # predicted classes (what the benchmark's plan does) is within 1 %
    assert ev["speedup_vs_default_geomean"] > 2.0, ev
    assert ev["regret_mean"] < 0.08 and ev["regret_top8_mean"] < 0.01, ev
