"""Schedule autotuning over the C ABI's exhaustive tuner (dtc_autotune).

The reference chooses balance / vector width / N split from a fixed table
per dataset (scripts/DTCSpMM/run_DTC_SpMM.py:10-30). Here every schedule the
kernels support is timed on the caller's own ME-TCF and B (``autotune``), and
``tune_forms`` extends the search over the B storage forms that meet an error
budget. A schedule changes neither the B form nor the product precision:
schedules of one form differ only in how fp32 partial sums are grouped (all
within the form's error bound), and each schedule is bitwise reproducible.
"""
import ctypes as C
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import (B_BF16, B_BF16X2, B_F32, B_FP8, B_SPLIT24, PREC_SPLIT3, PREC_SPLIT4,
                   PREC_TF32, Schedule, call)
from .metcf import METCF, _ptr, _stream, pack_b, spmm_ex

# name -> (B storage form, product precision, B bytes per element, relative
# error class vs FP64 on normalised inputs). The classes are the measured
# errors of the precision tests rounded up to a power of ten; a form is
# eligible under an error budget when its class is within it.
FORMS = {
    "tf32": (B_F32, PREC_TF32, 4.0, 1e-3),
    "split24x4": (B_SPLIT24, PREC_SPLIT4, 3.0, 1e-5),
    "split24x3": (B_SPLIT24, PREC_SPLIT3, 3.0, 1e-5),
    "bf16x2x3": (B_BF16X2, PREC_SPLIT3, 4.0, 1e-5),
    "bf16": (B_BF16, PREC_SPLIT4, 2.0, 1e-2),
    "fp8": (B_FP8, PREC_SPLIT4, 1.0, 1e-1),
}


def candidates(N, H=16, split=False):
    """Every (mode, waves, ntile) schedule the kernels support for width N at
    window height H (split: the split-precision kernels)."""
    L = _lib.lib()
    n = L.dtc_schedule_candidates_ex(N, H, 1 if split else 0, None, 0)
    arr = (Schedule * n)()
    L.dtc_schedule_candidates_ex(N, H, 1 if split else 0, arr, n)
    return list(arr)


def workspace_for(m: METCF, N, device):
    b = C.c_size_t()
    call("dtc_autotune_workspace_bytes", m.M, m.T, N, m.H, C.byref(b))
    return torch.empty(max(b.value, 1), dtype=torch.uint8, device=device)


def autotune(m: METCF, planes, fmt, N, precision, reps=3, use_values=True, out=None,
             workspace=None):
    """Times every candidate schedule; returns (list of measured Schedules, best)."""
    dev = planes[0].device
    C_ = out if out is not None else torch.empty((m.M, N), dtype=torch.float32, device=dev)
    ws = workspace if workspace is not None else workspace_for(m, N, dev)
    ncand = len(candidates(N, m.H, not (fmt == B_F32 and precision == PREC_TF32)))
    res = (Schedule * ncand)()
    nres, best = C.c_int(), C.c_int()
    vals = m.TCvalues if use_values else None
    call("dtc_autotune", _ptr(m.RowWindowOffset), _ptr(m.TCblocktileId), _ptr(m.TCblockoffset),
         _ptr(m.SparseAToX), _ptr(vals), m.M, m.nwin, m.T, m.H, m.W, fmt, _ptr(planes[0]),
         _ptr(planes[1]) if len(planes) > 1 else None, N, precision, _ptr(C_), _ptr(ws),
         ws.numel(), reps, res, ncand, C.byref(nres), C.byref(best), _stream())
    out_list = list(res)[: nres.value]
    return out_list, out_list[best.value]


def run(m: METCF, planes, fmt, N, precision, sched: Schedule, use_values=True, out=None,
        workspace=None):
    """SpMM with an explicit schedule (the tuned call)."""
    return spmm_ex(m, planes, fmt, N, precision, mode=sched.mode, grid=sched.grid,
                   use_values=use_values, out=out, workspace=workspace, ntile=sched.ntile)


@dataclass
class Choice:
    form: str
    schedule: Schedule
    ms: float


def eligible_forms(max_rel_err):
    return [k for k, v in FORMS.items() if v[3] <= max_rel_err]


def tune_forms(m: METCF, B: torch.Tensor, max_rel_err=1e-5, reps=3, forms=None):
    """Exhaustive search over (form within the error budget) x schedule.

    Returns (best Choice, {form: [measured Schedules]}) -- the table the
    learned cost model is trained on and evaluated against.
    """
    N = B.shape[1]
    forms = forms if forms is not None else eligible_forms(max_rel_err)
    if not forms:
        raise ValueError(f"no B form meets relative error {max_rel_err}")
    out = torch.empty((m.M, N), dtype=torch.float32, device=B.device)
    ws = workspace_for(m, N, B.device)
    table, best = {}, None
    for f in forms:
        fmt, prec = FORMS[f][0], FORMS[f][1]
        planes = [B.contiguous()] if fmt == B_F32 else pack_b(B, fmt)
        scheds, b = autotune(m, planes, fmt, N, prec, reps=reps, out=out, workspace=ws)
        table[f] = scheds
        if best is None or b.ms < best.ms:
            best = Choice(f, b, b.ms)
    return best, table
