"""losses_comp and print_lambda on the GPU (GPU tests): rtb_loss_ratios and
rtb_unique_lambdas against the oracle bit for bit, and the rt_loss_comp and
rt_print_lambda programs against the reference's own losses_comp and
print_lambda (oracle/_ref, compiled from their sources): the same bytes.
"""
import os
import subprocess

import numpy as np
import pytest
import torch

import loss_cases as LC
import pyoracle as O
from rt_b200 import engine as E
from rt_b200 import schemes as S
from test_losses import LOSSES, PRINT, bits_equal, read_blocks, synthetic_files

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "rt_b200", "bin")


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def all_files(d):
    return [LC.write_case(d, nm) for nm in sorted(LC.cases())] + synthetic_files(d)


def test_loss_ratios_equal_the_oracle(tmp_path):
    for f in all_files(str(tmp_path)):
        n, ng, nl, lam = LC.read_lambda(f)
        ll, ratio = E.loss_ratios(dev(lam), ng, nl)
        oll, oratio = O.loss_ratios(lam, ng, nl)
        assert bits_equal(ll, oll) and bits_equal(ratio, oratio), f
    # not a composite grid (windows that run over the good rays), nl = 0
    rng = np.random.default_rng(3)
    for lam, ng, nl in ((rng.choice([0.4, 0.5, 0.6], size=100), 40, 3), (np.array([0.5, 0.6]), 1, 3),
                        (rng.uniform(0.4, 0.7, size=1000), 600, 1000), (np.full(50, 0.55), 50, 1)):
        ll, ratio = E.loss_ratios(dev(lam), ng, nl)
        oll, oratio = O.loss_ratios(lam, ng, nl)
        assert bits_equal(ll, oll) and bits_equal(ratio, oratio)


def test_unique_lambdas_equal_the_oracle(tmp_path):
    for f in all_files(str(tmp_path)):
        n, ng, nl, lam = LC.read_lambda(f)
        got = E.unique_lambdas(dev(lam[:ng]), ng, max(nl, 1))
        assert bits_equal(got, O.unique_lambdas(lam, ng, 0)[:max(nl, 1)]), f   # 0: every distinct value
    lam = np.array([0.5, 0.6, 0.5, 0.7, 0.8, 0.6, np.nan, np.nan, -0.0, 0.0])
    assert bits_equal(E.unique_lambdas(dev(lam), len(lam), 100), O.unique_lambdas(lam, len(lam), 0))
    assert list(E.unique_lambdas(dev(lam), len(lam), 2)) == [0.5, 0.6]


def run(cmd, cwd):
    out = subprocess.run(cmd, cwd=str(cwd), capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    return out


@pytest.mark.skipif(not os.path.exists(LOSSES), reason="reference losses_comp not built")
def test_rt_loss_comp_equals_reference_losses_comp(tmp_path):
    files = synthetic_files(str(tmp_path))
    (tmp_path / "list.txt").write_text("".join(f + "\n" for f in files))
    run([LOSSES, "list.txt", "ref.bin"], tmp_path)
    run([os.path.join(BIN, "rt_loss_comp"), "list.txt", "ours.bin"], tmp_path)
    assert (tmp_path / "ours.bin").read_bytes() == (tmp_path / "ref.bin").read_bytes()


@pytest.mark.skipif(not os.path.exists(PRINT), reason="reference print_lambda not built")
def test_rt_print_lambda_equals_reference_print_lambda(tmp_path):
    files = all_files(str(tmp_path))
    (tmp_path / "list.txt").write_text("".join(f + "\n" for f in files))
    ref = run([PRINT, "list.txt"], tmp_path).stdout
    ours = run([os.path.join(BIN, "rt_print_lambda"), "list.txt"], tmp_path).stdout
    assert ours == ref and ref.count("#") == len(files)


def test_rt_trace_then_rt_loss_comp(tmp_path):
    """The echelle over three orders through rt_trace, then rt_loss_comp on
    its result list: each block is the oracle's, the last one twice (the
    list ends in a newline)."""
    ranges = [[0.38 + 0.001 * k, 0.9, m, 1] for k, m in enumerate((33, 45, 58))]
    xml = str(tmp_path / "c1s.xml")
    S.write_xml(xml, S.echelle(), "C1 small", "c1s", 300, S.C1_RADIUS, ranges, n_lambda=S.C1_NLAMBDA)
    run([os.path.join(BIN, "rt_trace"), xml, "rt_files.txt", "log.txt", "--seed", "5"], tmp_path)
    files = [ln.strip() for ln in open(tmp_path / "rt_files.txt") if ln.strip()]
    run([os.path.join(BIN, "rt_loss_comp"), "rt_files.txt", "losses.bin"], tmp_path)
    blocks = read_blocks(str(tmp_path / "losses.bin"))
    assert len(blocks) == len(files) + 1
    for k, f in enumerate(files + files[-1:]):
        n, ng, nl, lam = LC.read_lambda(str(tmp_path / f))
        ll, ratio = O.loss_ratios(lam, ng, nl)
        assert bits_equal(blocks[k][0], ll) and bits_equal(blocks[k][1], ratio)
