"""Per-CTA timing of the SpMM kernels: the load-balance report.

``cta_report(fn, capacity)`` turns on the library's per-CTA timer records
(dtc_set_cta_timer), runs ``fn`` once (one SpMM launch), turns them off and
summarises: for every CTA its busy time (kernel entry to exit, %globaltimer)
and chunk count, per SM the sum of its CTAs' busy time, and the launch span.
The reference instruments balance with separate per-SM clock kernels
(DTC-SpMM/DTCSpMM_kernel.cu:62-79, :1004-1018); here the product kernels
record it themselves behind a switch that is off by default.
"""
import ctypes as C

import numpy as np
import torch

from ._lib import call


def cta_records(fn, capacity=65536, device=None):
    """Runs fn() with per-CTA timing on; returns an int64 array [ctas, 4] of
    (entry ns, exit ns, SM id, chunks) for the CTAs that ran."""
    dev = torch.device("cuda") if device is None else device
    buf = torch.zeros(4 * capacity, dtype=torch.int64, device=dev)
    torch.cuda.synchronize(dev)
    call("dtc_set_cta_timer", C.c_void_p(buf.data_ptr()), capacity)
    try:
        fn()
        torch.cuda.synchronize(dev)
    finally:
        call("dtc_set_cta_timer", None, 0)
    rec = buf.view(capacity, 4).cpu().numpy()
    return rec[rec[:, 1] > 0]


def summarize(rec):
    """Busy-time statistics of one launch's CTA records (microseconds)."""
    if len(rec) == 0:
        return {"ctas": 0}
    t0 = rec[:, 0].min()
    entry, exit_ = (rec[:, 0] - t0) / 1e3, (rec[:, 1] - t0) / 1e3
    busy = exit_ - entry
    sm = rec[:, 2]
    sms = np.unique(sm)
    sm_busy = np.array([busy[sm == s].sum() for s in sms])
    return {"ctas": int(len(rec)), "sms": int(len(sms)), "span_us": float(exit_.max()),
            "cta_busy_us": {"mean": float(busy.mean()), "max": float(busy.max()),
                            "p10": float(np.percentile(busy, 10)),
                            "p90": float(np.percentile(busy, 90))},
            "sm_busy_us": {"mean": float(sm_busy.mean()), "max": float(sm_busy.max()),
                           "min": float(sm_busy.min())},
            "sm_imbalance": float(sm_busy.max() / sm_busy.mean()),
            "chunks_per_cta": {"mean": float(rec[:, 3].mean()), "max": int(rec[:, 3].max())},
            "last_exit_minus_first_exit_us": float(exit_.max() - exit_.min())}


def cta_report(fn, capacity=65536, device=None):
    return summarize(cta_records(fn, capacity, device))
