"""GPU tests of the NMF_GPU drop-in command line against the reference fixtures."""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR, load_golden, maxnorm_rel

pytestmark = pytest.mark.gpu
CLI = os.path.join(PKG_DIR, "NMF_GPU")


def run_cli(args, env_extra=None):
    env = dict(os.environ, NMFB_SEED="3")
    env.update(env_extra or {})
    p = subprocess.run([CLI] + args, capture_output=True, text=True, env=env, timeout=600)
    return p.returncode, p.stdout + p.stderr


@pytest.mark.parametrize("case", ["A_fixed50", "odd_37x19_k2", "r300x70_k5"])
def test_cli_binary_io_matches_reference(pkg, tmp_path, case):
    import nmf_b200.matrix_io as mio
    g = load_golden(case)
    fn = str(tmp_path / case)
    mio.save(fn, "dat", g["V"])
    k, it, j, t = (int(g[x]) for x in ("k", "n_iters", "niter_test_conv", "stop_threshold"))
    rc, out = run_cli([fn, "-b", "0", "-e", "0", "-k", str(k), "-i", str(it), "-j", str(j), "-t", str(t)])
    assert rc == 0, out
    m = re.search(r"NMF: Algorithm converged in (\d+) iterations\.", out) or \
        re.search(r"NMF: (\d+) iterations performed\.", out)
    assert int(m.group(1)) == int(g["iterations"])
    dist = float(re.search(r"Distance between V and W\*H: ([0-9.eE+-]+)", out).group(1))
    assert abs(dist - float(g["distance"])) <= 1e-5 * float(g["distance"]) + 5e-7
    W = mio.load(fn + "_W.dat", "dat")[0]
    Ht = mio.load(fn + "_H.dat", "dat")[0]          # written K x M, as the reference does
    assert W.shape == (g["V"].shape[0], k) and Ht.shape == (k, g["V"].shape[1])
    tol = 1e-4 if it <= 100 else 2e-3
    assert maxnorm_rel(W, g["W"]) < tol and maxnorm_rel(Ht.T, g["H"]) < tol


def test_cli_ascii_tagged_output(pkg, tmp_path):
    import nmf_b200.matrix_io as mio
    g = load_golden("odd_37x19_k2")
    V = g["V"]
    fn = str(tmp_path / "tagged.txt")
    mio.save(fn, "txt", V, name="Name", headers=[f"s{j}" for j in range(V.shape[1])],
             labels=[f"g{i}" for i in range(V.shape[0])])
    rc, out = run_cli([fn, "-k", "2", "-i", "30", "-j", "10"])
    assert rc == 0, out
    W, name, hdr, lbl = mio.load(fn + "_W.txt", "txt")
    assert name == "Name" and hdr == ["Factor_0", "Factor_1"] and lbl[:2] == ["g0", "g1"]
    Ht, name, hdr, lbl = mio.load(fn + "_H.txt", "txt")
    assert Ht.shape == (2, V.shape[1]) and lbl == ["Factor_0", "Factor_1"] and hdr[0] == "s0"
    assert maxnorm_rel(W, g["W"]) < 1e-4    # "%g" text output keeps 6 significant digits


def test_cli_rank_too_large(pkg, tmp_path):
    import nmf_b200.matrix_io as mio
    fn = str(tmp_path / "small.dat")
    mio.save(fn, "dat", np.ones((5, 3), np.float32))
    rc, out = run_cli([fn, "-b", "0", "-k", "4"])
    assert rc != 0 and "invalid factorization rank" in out
