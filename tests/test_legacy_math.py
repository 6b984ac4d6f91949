"""The identity behind floyd_min_plus_Nvidia of the legacy kernel ABI,
checked on the CPU in float32 (the arithmetic of the reference's CUDA
kernel): with E the min-plus identity (0 on the diagonal, 1e8 elsewhere),
[mat1 | E] (x) [mat2 ; res] from the sentinel equals min(res, mat1 (x) mat2)
for every res whose entries are at most 1e8, bit for bit."""
import numpy as np
import pytest

INF = np.float32(1e8)


def _minplus(A, B):
    C = np.full((A.shape[0], B.shape[1]), INF, np.float32)
    for k in range(A.shape[1]):
        C = np.minimum(C, A[:, k:k + 1] + B[k:k + 1, :])
    return C


@pytest.mark.parametrize("m,n,k", [(7, 5, 3), (1, 9, 0), (16, 16, 16), (23, 4, 31)])
@pytest.mark.parametrize("integral", [True, False])
def test_stacked_product_is_the_accumulating_update(m, n, k, integral):
    rng = np.random.default_rng(m * 100 + n * 10 + k + int(integral))

    def mat(r, c):
        x = (rng.integers(0, 60, (r, c)) if integral else rng.random((r, c)) * 60).astype(np.float32)
        x[rng.random((r, c)) < 0.3] = INF
        return x

    mat1, mat2, res = mat(m, k), mat(k, n), mat(m, n)
    E = np.full((m, m), INF, np.float32)
    np.fill_diagonal(E, 0)
    got = _minplus(np.hstack([mat1, E]), np.vstack([mat2, res]))
    want = np.minimum(res, _minplus(mat1, mat2))
    assert got.tobytes() == want.tobytes()
