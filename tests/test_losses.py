"""losses_comp and print_lambda (efficiency/losses_comp.cpp, tools/print_lambda.cpp)
without a GPU: the oracle's restatement against the reference's own programs,
compiled from their sources (oracle/_ref/losses_comp, oracle/_ref/print_lambda),
on result files of traced beams.
"""
import os
import subprocess

import numpy as np
import pytest

import loss_cases as LC
import pyoracle as O

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
LOSSES = os.path.join(REF, "losses_comp")
PRINT = os.path.join(REF, "print_lambda")


def read_blocks(path):
    blocks = []
    with open(path, "rb") as f:
        while True:
            h = f.read(8)
            if len(h) < 8:
                break
            (n,) = np.frombuffer(h, dtype=np.uint64)
            n = int(n)
            blocks.append((np.frombuffer(f.read(8 * n), dtype=np.float64),
                           np.frombuffer(f.read(8 * n), dtype=np.float64)))
    return blocks


def bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


SYNTH = [(64, 300, 1), (5, 2000, 2), (31, 97, 3), (1, 500, 4)]   # (n_lambda, rays per wavelength, seed)


def synthetic_files(d):
    files = []
    for nl, npl, seed in SYNTH:
        f = os.path.join(d, f"synth_{nl}_{npl}.dat")
        LC.write_synthetic(f, nl, npl, seed)
        files.append(f)
    return files


@pytest.mark.skipif(not os.path.exists(LOSSES), reason="reference losses_comp not built")
def test_oracle_matches_reference_losses_comp(tmp_path):
    """One block per listed file; a list ending in a newline repeats the last
    file's block (the reference reads names with >> until eof()).  The files
    keep every ray of their longest wavelength, so that no counting window
    runs past the good rays, where the reference reads beyond its array."""
    files = synthetic_files(str(tmp_path))
    (tmp_path / "list.txt").write_text("".join(f + "\n" for f in files))
    out = subprocess.run([LOSSES, "list.txt", "res.bin"], cwd=str(tmp_path), capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    blocks = read_blocks(str(tmp_path / "res.bin"))
    assert len(blocks) == len(files) + 1
    for k, f in enumerate(files + files[-1:]):
        n, ng, nl, lam = LC.read_lambda(f)
        ll, ratio = O.loss_ratios(lam, ng, nl)
        assert bits_equal(blocks[k][0], ll) and bits_equal(blocks[k][1], ratio), f
        # the transmitted share of each wavelength
        assert np.array_equal(ll, np.unique(lam))
        assert np.array_equal(np.round(ratio * (n // nl)), [np.sum(lam[:ng] == v) for v in ll])
    # a list without a final newline: no repeat
    (tmp_path / "list2.txt").write_text("\n".join(files))
    out = subprocess.run([LOSSES, "list2.txt", "res2.bin"], cwd=str(tmp_path), capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0 and len(read_blocks(str(tmp_path / "res2.bin"))) == len(files)


def test_oracle_loss_ratios_on_traced_beams(tmp_path):
    """Traced beams: ll are the beam's wavelengths and ratio each one's
    transmitted share."""
    for nm in sorted(LC.cases()):
        n, ng, nl, lam = LC.read_lambda(LC.write_case(str(tmp_path), nm))
        ll, ratio = O.loss_ratios(lam, ng, nl)
        assert np.array_equal(ll, np.unique(lam)), nm
        assert np.array_equal(np.round(ratio * (n // nl)), [np.sum(lam[:ng] == v) for v in ll]), nm


def test_oracle_loss_ratios_edge_cases():
    # wavelengths that are not a composite grid: windows that run over the good rays
    rng = np.random.default_rng(3)
    lam = rng.choice([0.4, 0.5, 0.6], size=100)
    ll, ratio = O.loss_ratios(lam, 40, 3)
    assert np.all(ratio >= 0) and ratio.sum() * 33 <= 40
    # more wavelengths than rays: nl = 0, the reference's 0/0
    ll, ratio = O.loss_ratios(np.array([0.5, 0.6]), 1, 3)
    assert np.all(np.isnan(ratio)) and np.all(ll == 0.5)


def fmt(name, values):
    return "# " + name + "\n" + "".join(f"{v:.9f}\n" for v in values) + "\n"


@pytest.mark.skipif(not os.path.exists(PRINT), reason="reference print_lambda not built")
def test_oracle_matches_reference_print_lambda(tmp_path):
    files = [LC.write_case(str(tmp_path), nm) for nm in sorted(LC.cases())] + synthetic_files(str(tmp_path))
    (tmp_path / "list.txt").write_text("".join(f + "\n" for f in files))
    out = subprocess.run([PRINT, "list.txt"], cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    expect = ""
    for f in files:
        n, ng, nl, lam = LC.read_lambda(f)
        expect += fmt(f, O.unique_lambdas(lam, ng, nl))
    assert out.stdout == expect


def test_oracle_unique_lambdas_stops_like_the_reference():
    lam = np.array([0.5, 0.6, 0.5, 0.7, 0.8])
    assert list(O.unique_lambdas(lam, 5, 2)) == [0.5, 0.6]
    assert list(O.unique_lambdas(lam, 5, 0)) == [0.5, 0.6, 0.7, 0.8]   # never reaches 0
    assert list(O.unique_lambdas(lam, 5, 1)) == [0.5, 0.6, 0.7, 0.8]   # passes 1 at the first step
    assert list(O.unique_lambdas(np.array([0.5, 0.5, 0.6]), 3, 1)) == [0.5]
