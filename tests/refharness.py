"""Runs oracle/_ref/harness_* (the reference's host classes over one engine).

Test infrastructure: writes the harness inputs (surface spec, injected beam,
table files) and reads its Beam::Save output (.dat, beam.cpp:636-715).
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

from rt_b200 import ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def harness(kind: str) -> str | None:
    p = os.path.join(REF_DIR, f"harness_{kind}")
    return p if os.path.exists(p) else None


def _index_token(t, d: str, name: str) -> str:
    if isinstance(t, (int, float)):
        return f"v:{float(t)!r}"
    path = os.path.join(d, name)
    with open(path, "w") as f:
        f.write("# lambda n\n")
        for x, y in zip(t[0], t[1]):
            f.write(f"{float(x)!r} {float(y)!r}\n")
    return "f:" + path


def write_spec(specs, orders, d: str) -> str:
    lines = [str(len(specs))]
    for k, s in enumerate(specs):
        params = list(s.params)
        t1 = _index_token(s.n1, d, f"n1_{k}.txt")
        t2 = _index_token(s.n2, d, f"n2_{k}.txt")
        size = list(s.size) + [0.0] * (2 - len(s.size))
        row = [s.cls, s.type, s.shape, s.grating_type, int(s.order), repr(float(s.gr_const)), len(params)]
        row += [repr(float(v)) for v in params]
        row += [repr(float(v)) for v in (size[0], size[1], s.center[0], s.center[1], *s.distance, *s.angles)]
        row += [t1, t2]
        lines.append(" ".join(str(v) for v in row))
    lines.append(" ".join([str(len(orders))] + [str(int(o)) for o in orders]))
    path = os.path.join(d, "spec.txt")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def write_beam(rays, d: str, sl=slice(None)) -> str:
    path = os.path.join(d, "beam.bin")
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", len(rays.X[sl])))
        for name in ("X", "Y", "Z", "cX", "cY", "cZ", "lambda_"):
            f.write(np.ascontiguousarray(getattr(rays, name)[sl], dtype=np.float64).tobytes())
    return path


def read_dat(path: str):
    """Beam::Save file -> (N, N_good, N_lambda, 7 x N array in file order)."""
    with open(path, "rb") as f:
        n, ng, nl = struct.unpack("<QQQ", f.read(24))
        good = np.frombuffer(f.read(7 * ng * 8), dtype=np.float64).reshape(7, ng)
        bad = np.frombuffer(f.read(7 * (n - ng) * 8), dtype=np.float64).reshape(7, n - ng)
    return n, ng, nl, np.concatenate([good, bad], axis=1)


def run_trace(kind: str, specs, orders, rays, sl=slice(None), timeout=600):
    """Run the harness; returns (exit code, parsed .dat or None)."""
    exe = harness(kind)
    if exe is None:
        raise FileNotFoundError(f"harness_{kind} not built")
    with tempfile.TemporaryDirectory() as d:
        spec = write_spec(specs, orders, d)
        beam = write_beam(rays, d, sl)
        out = os.path.join(d, "out.dat")
        p = subprocess.run([exe, "trace", spec, beam, out], capture_output=True, timeout=timeout)
        if p.returncode != 0 or not os.path.exists(out):
            return p.returncode, None
        return 0, read_dat(out)


def read_qe(path: str):
    """QE file (Scheme::ComputeQE, scheme.cpp:1318-1334) -> [(lambda, qe)]."""
    blocks = []
    with open(path, "rb") as f:
        while True:
            h = f.read(8)
            if len(h) < 8:
                break
            (n,) = struct.unpack("<Q", h)
            lam = np.frombuffer(f.read(8 * n), dtype=np.float64)
            qe = np.frombuffer(f.read(8 * n), dtype=np.float64)
            blocks.append((lam, qe))
    return blocks


def run_qe(kind: str, specs, rows, n_lambda: int, timeout=600):
    """ComputeQE's curves through the harness (the reference's Surface /
    Grating ApplyQE over one engine): specs are SurfaceSpec of the QE
    surfaces in scheme order.  Returns (exit code, blocks or None)."""
    exe = harness(kind)
    if exe is None:
        raise FileNotFoundError(f"harness_{kind} not built")
    rows = np.atleast_2d(np.asarray(rows, dtype=np.float64))
    with tempfile.TemporaryDirectory() as d:
        lines = [f"{n_lambda} {rows.shape[0]} {rows.shape[1]}"]
        lines += [" ".join(repr(float(v)) for v in r) for r in rows]
        lines.append(str(len(specs)))
        for k, s in enumerate(specs):
            row = [str(int(s.type)), _index_token(s.qe, d, f"qe_{k}.txt")]
            if s.type == ffi.GRATING:
                row += [str(int(s.order))] + [repr(float(v)) for v in (s.gr_const, s.alpha, s.gamma, s.blaze)]
                row += [str(len(s.rule_params))] + [repr(float(v)) for v in s.rule_params]
            lines.append(" ".join(row))
        spec = os.path.join(d, "qe_spec.txt")
        with open(spec, "w") as f:
            f.write("\n".join(lines) + "\n")
        out = os.path.join(d, "qe.bin")
        p = subprocess.run([exe, "qe", spec, out], capture_output=True, timeout=timeout)
        if p.returncode != 0 or not os.path.exists(out):
            return p.returncode, None
        return 0, read_qe(out)
