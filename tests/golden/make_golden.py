"""Generate the parity fixtures of tests/golden/ by running the reference itself.

Runs ``oracle/_ref/NMF_GPU`` -- NMF-mGPU's own single-GPU CUDA build compiled
from the reference sources by ``oracle/Makefile`` (``make -C oracle ref``) in
its parity mode: CPU_RANDOM (glibc srandom/random initialisation) and
FIXED_INIT (seed 3) -- on seeded synthetic inputs, reading back its binary
outputs (``-e 0``: little-endian float64) and its stdout.  Needs a GPU.

    python tests/golden/make_golden.py --out <directory> [--cases NAME ...]

Each case is written as ``<case>.npz`` holding the input V (float32; for
inputs above 200k entries only the generator call and the SHA-256 of V), the
reference's W (n x k) and H (m x k, un-transposed), the iteration count, the
"converged" flag, the printed Frobenius distance and the arguments used.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import os
import re
import struct
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "NMF_GPU")
SIG_REAL = 0xEDB10EA1


def _synth():
    spec = importlib.util.spec_from_file_location("nmfb_synth", os.path.join(ROOT, "bionmf-gpu_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def write_binary(path: str, V: np.ndarray):
    """Non-native binary matrix file (src/matrix_io/matrix_io.c:3701-3830 layout):
    u32 signature 0xEDB10EA1, u32 rows, u32 cols, rows*cols float64 (LE)."""
    n, m = V.shape
    with open(path, "wb") as f:
        f.write(struct.pack("<III", SIG_REAL, n, m))
        f.write(np.ascontiguousarray(V, dtype="<f8").tobytes())


def read_binary(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        sig, r, c = struct.unpack("<III", f.read(12))
        assert sig == SIG_REAL, hex(sig)
        data = np.frombuffer(f.read(8 * r * c), dtype="<f8").reshape(r, c)
    return data


CASES = {
    # name: (generator args, k, -i, -j, -t)
    "A_conv": (("config_a", {}), 3, 2000, 10, 40),
    "A_fixed50": (("config_a", {}), 3, 50, 100, 40),
    "D_k5_conv": (("config_d", {}), 5, 2000, 10, 40),
    "odd_37x19_k2": (("expression_like", dict(n=37, m=19, k=2, seed=11)), 2, 30, 10, 40),
    "r300x70_k5": (("expression_like", dict(n=300, m=70, k=5, seed=12)), 5, 200, 10, 5),
    "r200x60_k40": (("expression_like", dict(n=200, m=60, k=40, seed=13)), 40, 20, 5, 100),
    "r400x128_k100": (("expression_like", dict(n=400, m=128, k=100, seed=14)), 100, 10, 5, 100),
    "B_small_k16": (("expression_like", dict(n=2000, m=300, k=16, seed=15, dirichlet=2.0, zero_frac=0.01)),
                    16, 100, 10, 1000000),
    # the benchmarked config B matrix (20000 x 1000, k = 16, 1 % zeros) and the
    # 6000 x 500 submatrix of the precision comparison, fixed iteration counts
    "B_k16_fixed100": (("config_b", {}), 16, 100, 10, 1000000),
    "Csub_6000x500_k32": (("poisson_counts", dict(n=6000, m=500, k=32, seed=63)), 32, 50, 10, 1000000),
}


def make_input(synth, gen):
    name, kw = gen
    V, labels = getattr(synth, name)(**kw)
    return V, labels


def safe_input_path(tmp, name):
    """The reference allocates strlen(filename) + strlen(ext) bytes for the
    output name "<filename>_W<ext>" (src/NMF_GPU.c:975-990), three bytes short.
    Pick a path length whose malloc rounding leaves room for those bytes."""
    base = os.path.join(tmp, name)
    while True:
        s = len(base) + 4                      # what the reference passes to malloc
        chunk = max(32, (s + 8 + 15) & ~15)    # glibc chunk size
        if chunk - 8 >= s + 3:
            return base
        base += "_"


def run_case(name, spec, outdir, tmp):
    synth = _synth()
    (gen, k, it, j, t) = spec
    V, labels = make_input(synth, gen)
    fn = safe_input_path(tmp, name)
    write_binary(fn, V)
    cmd = [REF_BIN, fn, "-b", "0", "-e", "0", "-k", str(k), "-i", str(it), "-j", str(j), "-t", str(t)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    out = p.stdout + p.stderr
    if p.returncode != 0:
        raise RuntimeError(f"{name}: reference exited {p.returncode}:\n{out}")
    W = read_binary(fn + "_W.dat")            # n x k
    Ht = read_binary(fn + "_H.dat")           # k x m (written transposed)
    m_conv = re.search(r"converged in (\d+) iterations", out)
    m_perf = re.search(r"NMF: (\d+) iterations performed", out)
    iters = int(m_conv.group(1)) if m_conv else int(m_perf.group(1))
    dist = float(re.search(r"Distance between V and W\*H: ([0-9.eE+-]+)", out).group(1))
    gpu_t = re.search(r"GPU \+ classification \+ check_result time: ([0-9.eE+-]+)", out)
    fields = dict(labels=labels, W=W.astype(np.float32), H=np.ascontiguousarray(Ht.T).astype(np.float32),
                  iterations=iters, converged=bool(m_conv), distance=dist, k=k, n_iters=it, niter_test_conv=j,
                  stop_threshold=t, seed=3, stdout=out, generator=json.dumps([gen[0], gen[1]]),
                  v_sha256=hashlib.sha256(np.ascontiguousarray(V, np.float32).tobytes()).hexdigest())
    if V.size <= 200000:   # larger inputs are regenerated from the seeded generator
        fields["V"] = V
    np.savez_compressed(os.path.join(outdir, name + ".npz"), **fields)
    return dict(case=name, iterations=iters, converged=bool(m_conv), distance=dist,
                gpu_seconds=float(gpu_t.group(1)) if gpu_t else None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory for the <case>.npz fixtures and summary.json")
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    a = ap.parse_args()
    if not os.path.exists(REF_BIN):
        sys.exit(f"{REF_BIN} missing: run `make -C oracle ref` where the reference sources are present")
    os.makedirs(a.out, exist_ok=True)
    summary = []
    with tempfile.TemporaryDirectory() as tmp:
        for name in a.cases:
            r = run_case(name, CASES[name], a.out, tmp)
            print(json.dumps(r), flush=True)
            summary.append(r)
    with open(os.path.join(a.out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
