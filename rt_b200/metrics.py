"""Accuracy of a trace against a reference trace at the CCD.

Both traces are the same rays (same index) through the same scheme; the
reference is the plain FP64 engine (bit-identical to the FP64 oracle).
"""
from __future__ import annotations


def ccd_error(x, y, flag, x_ref, y_ref, flag_ref, xsize, ysize, xpix, ypix):
    """Error of CCD positions in micrometres over rays good in both, and the
    pixel-assignment mismatch rate over rays good in either (a ray counts as a
    mismatch if it is good in one trace only or lands on another pixel).
    Arguments are torch tensors (or numpy arrays) of the final X, Y (mm) and
    flags."""
    import torch
    t = lambda a: a if isinstance(a, torch.Tensor) else torch.as_tensor(a)
    x, y, flag, x_ref, y_ref, flag_ref = map(t, (x, y, flag, x_ref, y_ref, flag_ref))
    g, gr = flag == 1, flag_ref == 1
    both = g & gr
    err = torch.hypot(x[both] - x_ref[both], y[both] - y_ref[both]) * 1000.0
    either = int((g | gr).sum())
    pix = lambda X, Y: (torch.floor((X + xsize / 2.0) / xpix), torch.floor((Y + ysize / 2.0) / ypix))
    px, py = pix(x[both], y[both])
    rx, ry = pix(x_ref[both], y_ref[both])
    moved = int(((px != rx) | (py != ry)).sum())
    flag_diff = int((g ^ gr).sum())
    out = {"rays_compared": int(both.sum()), "flag_mismatch": flag_diff, "pixel_moved": moved,
           "pixel_mismatch_rate": (moved + flag_diff) / max(1, either)}
    if err.numel():
        e = err.double()
        q = torch.quantile(e[: 16_000_000], torch.tensor([0.5, 0.999], dtype=torch.float64, device=e.device))
        out.update(median_um=float(q[0]), p99_9_um=float(q[1]), max_um=float(e.max()))
    return out
