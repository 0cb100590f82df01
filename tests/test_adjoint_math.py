"""The adjoint arithmetic (cfd_inwsl_b200/csrc/adjoint_math.h) on the CPU.

The header is compiled by the host compiler (tests/adjoint_harness.cpp); each
hand-written vector-Jacobian product (WCNS5 interpolation, Roe flux, node
flux, the whole face: projection, interpolation, back projection, Roe) is
checked entry by entry against central finite differences of the same forward
formulas evaluated in long double. Tolerance 1e-6 relative to the Jacobian row.
TENO interpolations (TENO-Z, cut-off 1e-5; TENO-Cong, CT of Teno5_CongZ) are
differentiated with the cut-off decision frozen at the evaluation point; the
stencils below are away from decision boundaries, so finite differences see
the same selection.
"""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
LD = C.c_longdouble


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    out = tmp_path_factory.mktemp("adj") / "libadjh.so"
    subprocess.run([cxx, "-std=c++17", "-O2", "-shared", "-fPIC", "-I", str(ROOT / "cfd_inwsl_b200" / "csrc"),
                    str(ROOT / "tests" / "adjoint_harness.cpp"), "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    lib.h_wcns5_fwd.restype = LD
    lib.h_interp_fwd.restype = LD
    lib.h_interp_fwd.argtypes = [C.c_int, C.c_void_p, C.c_double]
    lib.h_interp_vjp.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_void_p]
    lib.h_teno_flag.restype = C.c_uint
    lib.h_teno_flag.argtypes = [C.c_int, C.c_void_p, C.c_double]
    lib.h_face_fwd_f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    lib.h_face_vjp_f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def ld(a):
    return (LD * len(a))(*[float(x) for x in a])


def dbl(a):
    return (C.c_double * len(a))(*[float(x) for x in a])


def fd_jacobian(fun, x, nout):
    J = np.zeros((nout, len(x)))
    for i in range(len(x)):
        e = 1e-7 * max(1.0, abs(x[i]))
        xp = np.array(x, dtype=np.longdouble)
        xm = xp.copy()
        xp[i] += e
        xm[i] -= e
        J[:, i] = ((np.array(fun(xp), dtype=np.longdouble) - np.array(fun(xm), dtype=np.longdouble)) /
                   (2 * np.longdouble(e))).astype(float)
    return J


def prim_to_cons(p):
    r, u, v, pp = p
    return [r, r * u, r * v, pp / 0.4 + 0.5 * r * (u * u + v * v)]


def check_rows(J, vjp_of_row):
    for k in range(J.shape[0]):
        g = vjp_of_row(k)
        assert np.abs(J[k] - g).max() <= 1e-6 * max(np.abs(J[k]).max(), 1e-12), (k, J[k], g)


def test_wcns5_vjp(harness):
    rng = np.random.default_rng(0)
    for scale in (1.0, 1e-2, 1e-3):
        q = rng.normal(size=5) * scale
        J = fd_jacobian(lambda x: [harness.h_wcns5_fwd(ld(x))], q, 1)
        qb = (C.c_double * 5)()
        harness.h_wcns5_vjp(dbl(q), C.c_double(1.0), qb)
        assert np.abs(J[0] - np.array(qb)).max() <= 1e-6 * np.abs(J[0]).max()


@pytest.mark.parametrize("ax", [0, 1])
def test_roe_vjp(harness, ax):
    rng = np.random.default_rng(1 + ax)
    cases = [([1.2, 0.5, 0.3, 0.8], [0.9, 0.45, 0.35, 0.7]),
             ([1.0, 0.02, -0.01, 1.0], [1.05, -0.01, 0.02, 1.1])]  # entropy fix active on the slow wave
    for _ in range(4):
        L = [rng.uniform(0.5, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.5, 2)]
        R = [rng.uniform(0.5, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.5, 2)]
        cases.append((L, R))
    for L, R in cases:
        def f(x):
            out = (LD * 4)()
            harness.h_roe_fwd(ax, ld(x[:4]), ld(x[4:]), out)
            return list(out)

        J = fd_jacobian(f, L + R, 4)

        def row(k):
            Fb = np.zeros(4)
            Fb[k] = 1.0
            Lb, Rb = (C.c_double * 4)(), (C.c_double * 4)()
            harness.h_roe_vjp(ax, dbl(L), dbl(R), dbl(Fb), Lb, Rb)
            return np.array(list(Lb) + list(Rb))

        check_rows(J, row)


@pytest.mark.parametrize("ax", [0, 1])
def test_node_vjp(harness, ax):
    U = prim_to_cons([1.1, 0.4, -0.2, 0.9])

    def f(x):
        out = (LD * 4)()
        harness.h_node_fwd(ax, ld(x), out)
        return list(out)

    J = fd_jacobian(f, U, 4)

    def row(k):
        Gb = np.zeros(4)
        Gb[k] = 1.0
        ub = (C.c_double * 4)()
        harness.h_node_vjp(ax, dbl(U), dbl(Gb), ub)
        return np.array(list(ub))

    check_rows(J, row)


@pytest.mark.parametrize("ax", [0, 1])
@pytest.mark.parametrize("kind", ["smooth", "rough"])
def test_face_vjp(harness, ax, kind):
    rng = np.random.default_rng(10 + ax)
    x = np.linspace(0, 1, 6)
    if kind == "smooth":
        prims = [[1 + 0.2 * np.sin(3 * xi + 0.3), 0.5 + 0.1 * np.cos(2 * xi), 0.3 + 0.05 * xi, 0.7 + 0.1 * np.sin(xi)]
                 for xi in x]
    else:
        prims = [[rng.uniform(0.5, 1.5), rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5), rng.uniform(0.5, 1.5)]
                 for _ in x]
    U6 = sum((prim_to_cons(p) for p in prims), [])

    def f(xx):
        out = (LD * 4)()
        harness.h_face_fwd(ax, ld(xx), out)
        return list(out)

    J = fd_jacobian(f, U6, 4)

    def row(k):
        Fb = np.zeros(4)
        Fb[k] = 1.0
        ub = (C.c_double * 24)()
        harness.h_face_vjp(ax, dbl(U6), dbl(Fb), ub)
        return np.array(list(ub))

    check_rows(J, row)


TENOZ, TENOCONG = 2, 3
CT = {TENOZ: 1e-5, TENOCONG: 0.15704178024750198}


@pytest.mark.parametrize("fam", [TENOZ, TENOCONG])
def test_teno_frozen_interpolation(harness, fam):
    """The frozen-flag TENO derivative is the selected stencil's coefficients;
    the stencils cover kept-all, one-cut and two-cut selections."""
    rng = np.random.default_rng(fam)
    seen = set()
    qs = [rng.normal(size=5) for _ in range(40)]
    # jumps with generic values (no smoothness indicator exactly zero: those
    # sit on a decision boundary)
    qs += [np.array([0.1, 0.12, 0.13, 1.0, 1.05]), np.array([1.0, 1.02, 0.1, 0.11, 0.125]),
           np.array([0.2, 0.21, 1.0, 1.03, 1.01]), np.array([1, 2, 3.1, 4, 5.2]),
           np.array([0.05, 0.0, 0.02, 0.01, 1.0])]
    for q in qs:
        flag = harness.h_teno_flag(fam, dbl(q), CT[fam])
        seen.add(flag)
        J = fd_jacobian(lambda x: [harness.h_interp_fwd(fam, ld(x), C.c_double(CT[fam]))], q, 1)
        qb = (C.c_double * 5)()
        harness.h_interp_vjp(fam, dbl(q), C.c_double(CT[fam]), C.c_double(1.0), qb)
        assert np.abs(J[0] - np.array(qb)).max() <= 1e-7 * np.abs(J[0]).max(), (q, flag, J[0], list(qb))
    assert 0 in seen and len(seen) >= 3, seen


@pytest.mark.parametrize("ax", [0, 1])
@pytest.mark.parametrize("fam", [TENOZ, TENOCONG])
@pytest.mark.parametrize("kind", ["smooth", "rough"])
def test_face_vjp_teno(harness, ax, fam, kind):
    rng = np.random.default_rng(20 + ax + 2 * fam)
    x = np.linspace(0, 1, 6)
    for trial in range(3):
        if kind == "smooth":
            ph = rng.uniform(0, 6)
            prims = [[1 + 0.2 * np.sin(3 * xi + ph), 0.5 + 0.1 * np.cos(2 * xi + ph), 0.3 + 0.05 * xi,
                      0.7 + 0.1 * np.sin(xi + ph)] for xi in x]
        else:
            prims = [[rng.uniform(0.5, 1.5), rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5), rng.uniform(0.5, 1.5)]
                     for _ in x]
        U6 = sum((prim_to_cons(p) for p in prims), [])

        def f(xx):
            out = (LD * 4)()
            harness.h_face_fwd_f(ax, fam, CT[fam], ld(xx), out)
            return list(out)

        J = fd_jacobian(f, U6, 4)

        def row(k):
            Fb = np.zeros(4)
            Fb[k] = 1.0
            ub = (C.c_double * 24)()
            harness.h_face_vjp_f(ax, fam, CT[fam], dbl(U6), dbl(Fb), ub)
            return np.array(list(ub))

        check_rows(J, row)
