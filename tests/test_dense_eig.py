"""The host linear algebra of the GMRES solver (topo-dda_b200/csrc/dense_eig.h:
Householder reduction, shifted QR, eigenvectors by back substitution and by
Hessenberg inverse iteration), compiled with g++ into a small harness and
checked against numpy on random, nearly triangular, graded and
deflated-restart-shaped matrices.  CPU only."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include "dense_eig.h"
#include <cstdio>
using namespace tdda;
int main() {
    int n, few;
    if (scanf("%d %d", &n, &few) != 2) return 1;
    DenseMat A(n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) { double a, b; if (scanf("%lf %lf", &a, &b) != 2) return 1; A(i, j) = {a, b}; }
    std::vector<cplx> ev; std::vector<std::vector<cplx>> V;
    auto all = [](const std::vector<cplx> &e) { std::vector<int> id; for (int i = 0; i < (int)e.size(); ++i) id.push_back(i); return id; };
    bool ok = few ? eigenpairs_few(A, ev, V, all) : eigenpairs(A, ev, V, all);
    printf("%d\n", ok ? 1 : 0);
    for (auto &e : ev) printf("%.17g %.17g\n", e.real(), e.imag());
    for (auto &v : V) for (auto &e : v) printf("%.17g %.17g\n", e.real(), e.imag());
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    d = tmp_path_factory.mktemp("eig")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "topo-dda_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)
    return str(exe)


def _run(exe, A, few):
    n = A.shape[0]
    inp = f"{n} {1 if few else 0}\n" + "\n".join(f"{float(A[i, j].real)!r} {float(A[i, j].imag)!r}"
                                                   for i in range(n) for j in range(n))
    out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    assert out[0] == "1"
    vals = np.array([complex(*map(float, l.split())) for l in out[1:1 + n + n * n]])
    return vals[:n], vals[n:].reshape(n, n).T


def _cases():
    rng = np.random.default_rng(5)
    for n in (1, 2, 5, 20, 60):
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        yield A
        yield np.triu(A) + 1e-3 * np.triu(A, -1) - 1e-3 * np.triu(A)  # nearly triangular
        yield A @ np.diag(np.geomspace(1e-6, 1, n)) @ np.linalg.inv(A + 3 * np.eye(n))  # graded
        k = max(1, n // 3)
        D = np.triu(A, -1)
        D[: k + 1, :k] = A[: k + 1, :k]  # Hessenberg with a dense leading block (a deflated restart)
        yield D


@pytest.mark.parametrize("few", [False, True])
def test_eigenpairs_match_numpy(harness, few):
    for A in _cases():
        ev, V = _run(harness, A, few)
        ref = np.linalg.eigvals(A)
        s = max(np.abs(ref).max(), 1e-300)
        assert max(min(abs(e - ref)) for e in ev) <= 1e-10 * s
        assert max(min(abs(r - ev)) for r in ref) <= 1e-10 * s
        res = np.linalg.norm(A @ V - V * ev[None, :], axis=0) / np.linalg.norm(A, 2)
        # inverse iteration on clustered eigenvalues converges more loosely
        assert res.max() <= (1e-8 if few else 1e-12), res.max()
