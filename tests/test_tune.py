"""Schedule autotuner (dtc_autotune): candidate enumeration on the host, and on
the GPU that every measured schedule computes the product within its form's
tolerance, that the chosen one is the fastest measured, and that re-running
it is bitwise reproducible."""
import numpy as np
import pytest

from dtc_b200 import tune


def test_candidates_cover_modes_waves_ntiles():
    c128 = tune.candidates(128)
    assert len(c128) == 7 + 5  # window mode 7 wave counts, balance mode 5; one N-tile
    assert {s.mode for s in c128} == {0, 1}
    assert {s.waves for s in c128 if s.mode == 0} == {1, 2, 4, 8, 16, 32, 64}
    assert {s.waves for s in c128 if s.mode == 1} == {1, 2, 4, 8, 16}
    assert {s.ntile for s in c128} == {1}
    c512 = tune.candidates(512)
    assert len(c512) == (7 + 5) * 3
    assert {s.ntile for s in c512} == {1, 2, 4}
    assert len({s.key() for s in c512}) == len(c512)
    assert tune.candidates(0) == []


def test_forms_by_error_budget():
    assert set(tune.eligible_forms(1e-5)) == {"split24x4", "split24x3", "bf16x2x3"}
    assert "tf32" in tune.eligible_forms(1e-3)
    assert tune.eligible_forms(1e-9) == []


def _bound_check(C, rp, col, val, M, B, tol):
    from oracle import oracle as O
    ref = O.spmm_f64(rp, col, val, M, B)
    bound = O.spmm_absbound_f64(rp, col, val, M, B)
    err = np.abs(C.astype(np.float64) - ref)
    assert (err <= tol * bound + 1e-6).all(), (err / (bound + 1e-30)).max()


@pytest.mark.gpu
@pytest.mark.parametrize("form,N", [("tf32", 128), ("split24x4", 256), ("split24x3", 128)])
def test_autotune_every_schedule_correct(cuda, form, N):
    import torch
    from dtc_b200 import gen, metcf
    A = gen.zipf(6000, seed=3)
    m = metcf.convert(A.rowptr, A.col, A.M, values=A.val)
    B = gen.normal(A.M, N, seed=4)
    Bd = torch.from_numpy(B).cuda()
    fmt, prec = tune.FORMS[form][0], tune.FORMS[form][1]
    planes = [Bd] if form == "tf32" else metcf.pack_b(Bd, fmt)
    scheds, best = tune.autotune(m, planes, fmt, N, prec, reps=2)
    assert len(scheds) == len(tune.candidates(N))
    assert best.ms == min(s.ms for s in scheds) and best.ms > 0
    tol = 2.0 ** -9 if form == "tf32" else 2.0 ** -14
    for s in scheds:
        assert s.grid >= 1
        C = tune.run(m, planes, fmt, N, prec, s).cpu().numpy()
        _bound_check(C, A.rowptr, A.col, A.val, A.M, B, tol)
    a = tune.run(m, planes, fmt, N, prec, best).cpu().numpy()
    b = tune.run(m, planes, fmt, N, prec, best).cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert metcf.device_status(clear=True) == 0


@pytest.mark.gpu
def test_tune_forms_picks_within_budget(cuda):
    import torch
    from dtc_b200 import gen, metcf
    A = gen.uniform(4096, mean=12, seed=1)
    m = metcf.convert(A.rowptr, A.col, A.M, values=A.val)
    B = torch.from_numpy(gen.normal(A.M, 128, seed=2)).cuda()
    best, table = tune.tune_forms(m, B, max_rel_err=1e-5, reps=1)
    assert set(table) == {"split24x4", "split24x3", "bf16x2x3"}
    assert best.form in table
    assert best.ms == min(s.ms for v in table.values() for s in v)
