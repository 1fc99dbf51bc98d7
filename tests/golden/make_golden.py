"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Runs only where the reference sources are present (they are not on the GPU
machines); the outputs are committed.
  * rhs_*.txt      generate_zero_sum_vector / generate_random_vector
                   (gpu_implementation/solver.hpp:29-61) compiled from the
                   reference header by ref_rhs_harness.cu;
  * <case>.mtx + <case>/l_sol.mtx + <case>/sol_diag.txt
                   the reference CPU factor (cpu_implementation/driver_local.cpp)
                   run with 1 thread and its std::random_device pinned to
                   RCHOL_REF_SEED (oracle/_ref/rchol_ref_cpu_pinned), so the
                   oracle's replay mode can be checked against it exactly.
Inputs are built here with numpy (log-uniform or unit weights, ascending-nnz
order with a seeded tie-break, a ground vertex appended for SDDM inputs).
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("RCHOL_REFERENCE", "/root/reference")
sys.path.insert(0, os.path.join(REPO, "oracle"))
import pyoracle as O  # noqa: E402


def grid_edges(dims):
    idx = np.arange(int(np.prod(dims))).reshape(dims[::-1])
    a, b = [], []
    for ax in range(len(dims)):
        sl0 = [slice(None)] * len(dims)
        sl1 = [slice(None)] * len(dims)
        sl0[ax] = slice(0, -1)
        sl1[ax] = slice(1, None)
        a.append(idx[tuple(sl0)].ravel())
        b.append(idx[tuple(sl1)].ravel())
    return int(np.prod(dims)), np.concatenate(a), np.concatenate(b)


def laplacian(dims, rng, log_weights=True, excess_frac=0.0):
    n, a, b = grid_edges(dims)
    w = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), len(a))) if log_weights else np.ones(len(a))
    deg = np.bincount(a, minlength=n) + np.bincount(b, minlength=n)
    perm = rng.permutation(n)
    order = perm[np.argsort(deg[perm], kind="stable")]
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    a2, b2 = inv[a], inv[b]
    wd = np.zeros(n)
    np.add.at(wd, a2, w)
    np.add.at(wd, b2, w)
    exc = np.zeros(n)
    if excess_frac > 0:
        pick = rng.random(n) < excess_frac
        exc[pick] = rng.uniform(0, 1e-1, pick.sum()) * wd[pick]
    rows = [a2, b2, np.arange(n)]
    cols = [b2, a2, np.arange(n)]
    vals = [-w, -w, wd + exc]
    N = n
    if (exc > 0).any():
        g = np.nonzero(exc > 0)[0]
        rows += [g, np.full(len(g), n), np.array([n])]
        cols += [np.full(len(g), n), g, np.array([n])]
        vals += [-exc[g], -exc[g], np.array([exc.sum()])]
        N = n + 1
    return N, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), N != n


def main():
    meta = {"reference": "Tianyu-Liang/Parallel-Randomized-Cholesky", "cases": {}, "rhs": {}}
    # ---- right-hand sides from the reference's own generators
    exe = os.path.join("/tmp", "rchol_ref_rhs")
    subprocess.run(["nvcc", "-std=c++17", "-I" + REF, "-I" + os.path.join(REPO, "oracle", "ref_shim"),
                    "-o", exe, os.path.join(HERE, "ref_rhs_harness.cu"), "-lcusparse", "-lcublas"], check=True)
    for n, seed, kind in [(7, 0, 0), (1000, 0, 0), (1000, 0, 1), (1000, 5, 0)]:
        out = subprocess.run([exe, str(n), str(seed), str(kind)], check=True, capture_output=True, text=True).stdout
        name = f"rhs_{'zerosum' if kind == 0 else 'uniform'}_n{n}_s{seed}.txt"
        with open(os.path.join(HERE, name), "w") as f:
            f.write(out)
        meta["rhs"][name] = dict(n=n, seed=seed, generator=["generate_zero_sum_vector",
                                                              "generate_random_vector"][kind])
    # ---- reference factor, seed-pinned, 1 thread
    cases = [
        ("grid16_logw", dict(dims=(16, 16), log_weights=True), 11, 0),
        ("grid12_unit", dict(dims=(12, 12), log_weights=False), 12, 0),
        ("cube8_sddm", dict(dims=(8, 8, 8), log_weights=True, excess_frac=0.05), 13, 1),
    ]
    for name, spec, seed, physics in cases:
        rng = np.random.default_rng(seed)
        N, r, c, v, ground = laplacian(spec["dims"], rng, spec["log_weights"], spec.get("excess_frac", 0.0))
        mtx = os.path.join(HERE, name + ".mtx")
        O.write_mtx(mtx, N, r, c, v)
        d = os.path.join(HERE, name)
        os.makedirs(d, exist_ok=True)
        env = dict(os.environ, OMP_NUM_THREADS="1", RCHOL_REF_SEED=str(seed))
        args = [O.REF_BIN_PINNED, mtx, "1", d + "/"] + (["1"] if physics else [])
        p = subprocess.run(args, env=env, capture_output=True, text=True, check=True)
        nnz_line = [ln for ln in p.stdout.splitlines() if ln.startswith("nnz ratio")]
        meta["cases"][name] = dict(n=N, pinned_seed=seed, physics=physics, ground=bool(ground),
                                   spec={k: list(x) if isinstance(x, tuple) else x for k, x in spec.items()},
                                   command=" ".join(["rchol_ref_cpu_pinned", name + ".mtx", "1", name + "/"] +
                                                    (["1"] if physics else [])),
                                   ref_stdout_nnz=nnz_line[0] if nnz_line else "")
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
