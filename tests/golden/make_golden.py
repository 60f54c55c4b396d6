"""Generates tests/golden/lu_cases.npz: seeded inputs with LAPACK getrf outputs.

The reference ships no golden vectors (its tests are property checks on Julia
RNG matrices that cannot be regenerated without Julia).  Its own pivot test
asserts that OxiBLAS's partial-pivot choices equal LAPACK getrf's for real
data (test/lapack/lapack_dense.jl:12-14: `F.p == LA.lu(A; check=false).p`).
These fixtures therefore record, for seeded numpy inputs of the reference's
test shapes (lapack_dense.jl:9, factorizations.jl:2) and its special cases
(singular column, graded columns, nearly singular), the interchange sequence
and factors of LAPACK dgetrf through scipy (OpenBLAS).  The oracle and the GPU
path are checked against them.

Run: python tests/golden/make_golden.py   (needs scipy; writes lu_cases.npz)
"""
import os

import numpy as np
import scipy
import scipy.linalg as sl

SEED = 0x0B1A5  # the reference test suite's seed value (test/testsetup.jl:5)


def cases():
    rng = np.random.default_rng(SEED)
    out = []
    for (m, n, bs) in ((1, 1, 32), (5, 5, 1), (17, 17, 16), (33, 20, 16), (20, 33, 16), (64, 64, 32),
                       (130, 97, 32), (97, 130, 64), (257, 257, 32), (13, 7, 7),
                       (7, 13, 7), (67, 65, 32), (65, 67, 32)):
        out.append((f"randn_{m}x{n}_bs{bs}", rng.standard_normal((m, n)), bs))
    # the reference also runs 257x257 at blocksize 64: same matrix, other blocking
    out.append(("randn_257x257_bs64", out[8][1], 64))
    A = rng.standard_normal((40, 40))
    A[:, 22] = 0.0  # column 23 (1-based) exactly zero: info == 23
    out.append(("singular_col23_40", A, 128))
    G = rng.standard_normal((80, 80)) @ np.diag(10.0 ** np.linspace(0, -12, 80))
    out.append(("graded_80", G, 128))
    N = rng.standard_normal((60, 60))
    N[:, -1] = N[:, 0] + np.finfo(float).eps * rng.standard_normal(60)
    out.append(("nearly_singular_60", N, 128))
    D = rng.standard_normal((128, 128)) + 128 * np.eye(128)
    out.append(("diagdominant_128", D, 128))
    return out


def main():
    data = {}
    names = []
    for name, A, bs in cases():
        lu, piv = sl.lu_factor(A, check_finite=False)
        q = min(A.shape)
        info = 0
        d = np.diag(lu)[:q]
        z = np.nonzero(d == 0)[0]
        if len(z):
            info = int(z[0]) + 1
        if name == "randn_257x257_bs64":
            data[f"{name}/same_as"] = np.array("randn_257x257_bs32")
        else:
            data[f"{name}/A"] = A
        data[f"{name}/ipiv"] = (piv[:q] + 1).astype(np.int64)
        # factors kept whole for the small cases, as a norm for the large ones
        if A.size <= 20000:
            data[f"{name}/lu"] = lu
        data[f"{name}/lu_fro"] = np.float64(np.linalg.norm(lu))
        data[f"{name}/bs"] = np.int64(bs)
        data[f"{name}/info"] = np.int64(info)
        names.append(name)
    data["names"] = np.array(names)
    data["generator"] = np.array(f"scipy {scipy.__version__} lu_factor (LAPACK dgetrf), numpy "
                                 f"{np.__version__} default_rng({SEED})")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lu_cases.npz")
    np.savez_compressed(path, **data)
    print(path, os.path.getsize(path), "bytes,", len(names), "cases")


if __name__ == "__main__":
    main()
