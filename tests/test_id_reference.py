"""CPU: the host ID restatement (``structure.interpolative_decomposition``), which checks the
GPU's batched ID, against the reference's own ``decomposition``
(matroxTest-V1/compression.h:446-523) compiled into oracle/_ref: same rank, same skeleton
columns, same P (both call the same OpenBLAS dgeqp3 / dtrsm, so the match is exact here; the
test allows 1e-13 of the largest entry).  The reference asserts nrows > ncols and fixes its
maximum rank at 256, so the cases respect both."""
import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import structure as S

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference library (oracle/_ref) not built")


def cases():
    rng = np.random.default_rng(7)
    X = S.gaussian_mixture(3000, 6, 5, -2.0, 2.0, 0.3, 1.0, seed=3)
    mats = []
    for nr, nc, kind, h in ((256, 64, "gaussian", 1.0), (512, 256, "gaussian", 2.0), (400, 128, "imq", 1.5),
                            (300, 150, "gaussian", 0.5), (97, 33, "imq", 3.0), (600, 300, "gaussian", 1.0),
                            (100, 40, "newton", 1.0)):
        idx = rng.choice(X.shape[0], nr + nc, replace=False)
        mats.append(S.kernel_matrix(X, idx[:nr], idx[nr:], S.KernelSpec(kind, h)))
    mats.append(rng.standard_normal((200, 5)) @ rng.standard_normal((5, 60)))  # exact rank 5
    mats.append(np.zeros((40, 12)))
    mats.append(rng.standard_normal((30, 1)))
    return mats


@pytest.mark.parametrize("tol", [1e-3, 1e-5, 1e-7])
def test_host_id_matches_reference_decomposition(tol):
    for b, m in enumerate(cases()):
        rp, rP = O.ref_decomposition(m, tol)
        hp, hP = S.interpolative_decomposition(np.asfortranarray(m), tol, 256)
        assert np.array_equal(rp, hp), (b, len(rp), len(hp))
        assert rP.shape == hP.shape
        assert float(np.abs(rP - hP).max()) <= 1e-13 * max(1.0, float(np.abs(rP).max())), b
