"""The Q2 generator with a refined ball (structured_q2_ball): the hanging-node
maps, the condensed operator and the transfer checked through properties that
hold for any correct construction (no reference mesh has this numbering)."""
import numpy as np
import pytest
import scipy.sparse as sp

from gascoignelib_b200.problem import structured_q2_ball
from oracle.oracle import Oracle


@pytest.fixture(scope="module")
def ball():
    return structured_q2_ball(2, 3, eps=1.0, beta=None)


def _masks(L):
    A = sp.csr_matrix((L.val, L.col, L.rowptr), shape=(L.n, L.n))
    S = sp.csr_matrix((np.ones_like(L.val), L.col, L.rowptr), shape=(L.n, L.n))
    dm = np.zeros(L.n, bool)
    dm[L.dirichlet] = True
    hm = np.zeros(L.n, bool)
    hm[L.hn_edges[:, 0]] = True
    hm[L.hn_faces[:, 0]] = True
    touch = np.asarray(S[:, np.nonzero(dm)[0]].sum(axis=1)).ravel() > 0
    return A, dm, hm, ~dm & ~hm & ~touch


def test_ball_refines_and_hangs(ball):
    L = ball.finest
    assert ball.nlevels == 4 and L.n > ball.levels[-2].n
    assert L.hn_edges.shape[0] > 0 and L.hn_faces.shape[0] > 0 and L.hn_disc == 3
    hang = np.concatenate([L.hn_edges[:, 0], L.hn_faces[:, 0]])
    assert np.unique(hang).size == hang.size
    parents = np.concatenate([L.hn_edges[:, 1:].ravel(), L.hn_faces[:, 1:].ravel()])
    assert not np.isin(parents, hang).any()
    # hanging nodes sit on coarse edges / faces: their parents are even nodes
    assert np.all(np.round(L.coord[parents] * 2 * 16) % 2 == 0)


def test_condensed_diffusion_is_symmetric_and_consistent(ball):
    L = ball.finest
    A, dm, hm, inner = _masks(L)
    assert inner.sum() > 1000
    assert abs(A - A.T).max() < 1e-14
    x, y, z = L.coord.T
    for f in (np.ones_like(x), x, y * z, x * y * z):   # harmonic: A f = 0 inside
        v = np.where(hm, 0.0, f)
        assert np.abs(A @ v)[inner].max() < 1e-13
    # hanging rows are identity rows, hanging columns empty elsewhere
    Ah = A[np.nonzero(hm)[0]]
    assert np.array_equal(Ah.nonzero()[1], np.sort(np.nonzero(hm)[0]))


def test_hanging_maps_reproduce_triquadratics(ball):
    L = ball.finest
    x, y, z = L.coord.T
    u = (1 + x - 2 * x ** 2) * (0.5 + y + y ** 2) * (1 - z ** 2) + (x * y * z) ** 2 - x * y * z
    v = u.copy()
    v[L.hn_edges[:, 0]] = 7.0
    v[L.hn_faces[:, 0]] = -3.0
    O = Oracle(ball, omega=0.3)
    assert np.abs(O.hn("average", ball.nlevels - 1, v) - u).max() < 1e-14


def test_transfer_to_ball_level_is_trilinear_exact(ball):
    T, Lc, L = ball.transfers[-1], ball.levels[-2], ball.finest
    g = lambda c: 1.0 + 2.0 * c[:, 0] - c[:, 1] + 3.0 * c[:, 2] + c[:, 0] * c[:, 1] * c[:, 2]
    uc = g(Lc.coord)
    uf = np.full(L.n, np.nan)
    uf[T.c2f] = uc
    for m in (T.zweier, T.vierer, T.achter):
        uf[m[:, 0]] = uc[m[:, 1:]].mean(axis=1)
    assert not np.isnan(uf).any()
    assert np.abs(uf - g(L.coord)).max() < 1e-14
