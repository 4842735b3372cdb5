"""Host-side checks of the symbolic analysis (no GPU needed).

The structure produced by the C++ nested dissection is verified directly
(permutation, update sets, extend-add maps, entry scatter), and the dense
supernodal algorithm the CUDA kernels implement is replayed in numpy on those
arrays: fronts assembled from the 7-point stencil, partial LU, explicit
triangular inverses, then the chained forward/backward and transposed
sweeps.  The replay must reproduce scipy's sparse solves of A x = b and
A^T x = b, which pins the ordering, the update sets and the solve algebra.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from orbit_b200.symbolic import Symbolic
from orbit_b200 import synthetic
from oracle import assembly


def _stencil_of(A, nz, ny, nx):
    """[7][N] stencil of a 7-point CSR matrix (centre, W, E, S, N, B, T)."""
    N = nz * ny * nx
    A = A.tocsr()
    st = np.zeros((7, N))
    off = [0, -1, 1, -nx, nx, -nx * ny, nx * ny]
    for c in range(N):
        k, r = divmod(c, nx * ny)
        j, i = divmod(r, nx)
        ok = [True, i > 0, i < nx - 1, j > 0, j < ny - 1, k > 0, k < nz - 1]
        for d in range(7):
            if ok[d]:
                st[d, c] = A[c, c + off[d]]
    return st


def _matrix(nz, ny, nx, seed=3):
    rng = np.random.default_rng(seed)
    g = synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=2000.0, rho_profile=True, cmfmc_frac=0.4)
    T = assembly.transport_block(g)
    d = rng.uniform(1e-6, 1e-4, nz * ny * nx)
    L = assembly.species_operator(T, d)
    return (sp.eye(nz * ny * nx) + 10800.0 * L).tocsr()


def _replay(sym, stencil):
    a = {k: sym.array(k) for k in ("perm", "first", "n", "m", "parent", "level", "child", "uoff",
                                   "uidx", "rel", "ldf", "front_off", "level_front_size",
                                   "ent_level_off", "ent_pos", "ent_src", "ginv", "ginv_off")}
    ns = len(a["n"])
    nlev = int(a["level"].max()) + 1
    flat = stencil.reshape(-1)
    fronts, fac = {}, {}
    for lev in range(nlev - 1, -1, -1):
        buf = np.zeros(a["level_front_size"][lev])
        e0, e1 = a["ent_level_off"][lev], a["ent_level_off"][lev + 1]
        buf[a["ent_pos"][e0:e1]] = flat[a["ent_src"][e0:e1]]
        for s in np.nonzero(a["level"] == lev)[0]:
            n, m, ld = int(a["n"][s]), int(a["m"][s]), int(a["ldf"][s])
            F = buf[a["front_off"][s]:a["front_off"][s] + (n + m) * ld].reshape(n + m, ld)[:, :n + m].copy()
            # gather form of the extend-add (as the assembly kernel does it):
            # F[i, j] += S_c[inv_c[i], inv_c[j]] wherever both are mapped
            w = n + m
            inv = a["ginv"][a["ginv_off"][s]:a["ginv_off"][s] + 2 * w].reshape(2, w)
            for q, c in enumerate(a["child"][2 * s:2 * s + 2]):
                if c < 0:
                    continue
                Sc = fronts.pop(c)
                rows = np.nonzero(inv[q] >= 0)[0]
                F[np.ix_(rows, rows)] += Sc[np.ix_(inv[q][rows], inv[q][rows])]
            F11, F12, F21, F22 = F[:n, :n], F[:n, n:], F[n:, :n], F[n:, n:]
            Lw = np.eye(n)
            U = F11.copy()
            for k in range(n):  # unpivoted LU
                Lw[k + 1:, k] = U[k + 1:, k] / U[k, k]
                U[k + 1:, k:] -= np.outer(Lw[k + 1:, k], U[k, k:])
            U = np.triu(U)
            Li, Ui = np.linalg.inv(Lw), np.linalg.inv(U)
            L21 = F21 @ Ui
            U12 = Li @ F12
            fronts[s] = F22 - L21 @ U12
            fac[s] = (np.tril(Li, -1) + np.triu(Ui), -L21 @ Li, -Ui @ U12)
    return a, fac


def _solve(a, fac, b, trans):
    ns = len(a["n"])
    nlev = int(a["level"].max()) + 1
    perm = a["perm"]
    bp = b[perm]
    y = np.zeros_like(bp)
    x = np.zeros_like(bp)
    W = {}
    for lev in range(nlev - 1, -1, -1):
        for s in np.nonzero(a["level"] == lev)[0]:
            n, m, f0 = int(a["n"][s]), int(a["m"][s]), int(a["first"][s])
            SQ, Pb, Qr = fac[s]
            v = np.zeros(n + m)
            v[:n] = bp[f0:f0 + n]
            for c in a["child"][2 * s:2 * s + 2]:
                if c >= 0:
                    v[a["rel"][a["uoff"][c]:a["uoff"][c + 1]]] += W.pop(c)
            if not trans:
                y[f0:f0 + n] = v[:n] + np.tril(SQ, -1) @ v[:n]
                W[s] = v[n:] + Pb @ v[:n]
            else:
                y[f0:f0 + n] = np.triu(SQ).T @ v[:n]
                W[s] = v[n:] + Qr.T @ v[:n]
    for lev in range(nlev):
        for s in np.nonzero(a["level"] == lev)[0]:
            n, m, f0 = int(a["n"][s]), int(a["m"][s]), int(a["first"][s])
            SQ, Pb, Qr = fac[s]
            xu = x[a["uidx"][a["uoff"][s]:a["uoff"][s + 1]]]
            if not trans:
                x[f0:f0 + n] = np.triu(SQ) @ y[f0:f0 + n] + Qr @ xu
            else:
                x[f0:f0 + n] = (np.tril(SQ, -1) + np.eye(n)).T @ y[f0:f0 + n] + Pb.T @ xu
    out = np.empty_like(x)
    out[perm] = x
    return out


@pytest.mark.parametrize("shape,leaf", [((3, 4, 5), 4), ((5, 7, 6), 16), ((4, 9, 11), 8)])
def test_structure(shape, leaf):
    sym = Symbolic(*shape, leaf_cells=leaf)
    N = sym.N
    perm = sym.array("perm")
    assert sorted(perm.tolist()) == list(range(N))
    n, m, first = sym.array("n"), sym.array("m"), sym.array("first")
    assert n.sum() == N and first[0] == 0 and np.all(np.diff(first) == n[:-1])
    par, uoff, uidx = sym.array("parent"), sym.array("uoff"), sym.array("uidx")
    assert (par < 0).sum() == 1
    for s in range(len(n)):
        u = uidx[uoff[s]:uoff[s + 1]]
        assert np.all(np.diff(u) > 0)
        assert np.all(u >= first[s] + n[s])  # only later (ancestor) unknowns
    assert sym.lunz == int((n.astype(np.int64) ** 2 + 2 * n.astype(np.int64) * m).sum())
    child, rel, ginv, goff = sym.array("child"), sym.array("rel"), sym.array("ginv"), sym.array("ginv_off")
    # extend-add maps increase (the solve's gathers stop at the first entry past a chunk)
    for s in range(len(n)):
        assert np.all(np.diff(rel[uoff[s]:uoff[s + 1]]) > 0)
    # inverse extend-add maps: ginv[s][q][rel_c[u]] == u for child q, -1 elsewhere
    for s in range(len(n)):
        w = int(n[s] + m[s])
        inv = ginv[goff[s]:goff[s] + 2 * w].reshape(2, w)
        for q in range(2):
            c = child[2 * s + q]
            expect = np.full(w, -1)
            if c >= 0:
                expect[rel[uoff[c]:uoff[c + 1]]] = np.arange(uoff[c + 1] - uoff[c])
            assert np.array_equal(inv[q], expect)


@pytest.mark.parametrize("shape,leaf", [((3, 4, 5), 4), ((5, 7, 6), 16), ((4, 9, 11), 8)])
def test_replay_matches_sparse_solve(shape, leaf):
    A = _matrix(*shape)
    st = _stencil_of(A, *shape)
    sym = Symbolic(*shape, leaf_cells=leaf)
    a, fac = _replay(sym, st)
    rng = np.random.default_rng(1)
    b = rng.standard_normal(sym.N)
    x = _solve(a, fac, b, trans=False)
    xr = spla.spsolve(A.tocsc(), b)
    assert np.abs(x - xr).max() <= 1e-11 * np.abs(xr).max()
    xt = _solve(a, fac, b, trans=True)
    xtr = spla.spsolve(A.T.tocsc(), b)
    assert np.abs(xt - xtr).max() <= 1e-11 * np.abs(xtr).max()


def test_config_shapes_fill():
    """Fill of the geometric dissection at the benchmark shapes (vs AMD 1.30 M / 45.7 M)."""
    s0 = Symbolic(15, 20, 24)
    s1 = Symbolic(15, 72, 80)
    assert s0.lunz < 2.5e6
    assert s1.lunz < 60e6
    assert s1.info["max_front"] < 2048


def _fused_count(sym, max_n=64):
    """Supernodes the analysis hands to the one-CTA front kernel: pivots
    0 < n <= max_n, an update set (m > 0), and the kernel's shared memory
    (inverses and their transpose, both panels, the pivot exchange slots)
    within 28,672 elements."""
    n = sym.array("n").astype(np.int64)
    m = sym.array("m").astype(np.int64)
    ldq = (n + 3) // 4 * 4 + 4
    ldl = (m + 3) // 4 * 4
    elems = 2 * n * ldq + 2 * n * ldl + 512
    return int(((m > 0) & (n > 0) & (n <= max_n) & (elems <= 28672)).sum())


@pytest.mark.parametrize("env,max_n", [(None, 64), ("32", 32), ("0", 0)])
def test_fused_front_selection(monkeypatch, env, max_n):
    if env is None:
        monkeypatch.delenv("ORBIT_B200_FUSED_MAX_N", raising=False)
    else:
        monkeypatch.setenv("ORBIT_B200_FUSED_MAX_N", env)
    for shape, leaf in (((15, 72, 80), 80), ((8, 22, 26), 48)):
        sym = Symbolic(*shape, leaf_cells=leaf)
        assert sym.info["fused_fronts"] == _fused_count(sym, max_n)
    if max_n == 64:
        # at the benchmark shape the three deepest levels are one-CTA fronts
        sym = Symbolic(15, 72, 80, leaf_cells=80)
        lev = sym.array("level")
        assert sym.info["fused_fronts"] == 1792
        assert np.all(sym.array("n")[lev >= lev.max() - 2] <= 64)


def test_front_algebra_through_inverse_of_f11():
    """The one-CTA fronts and the tensor-core pipeline form the panels through
    X = inv(U11) inv(L11) = inv(F11): Pb = -F21 X, Qr = -X F12, and the Schur
    complement F22 + Pb F12; the blocked CUDA-core path forms L21 = F21 inv(U11),
    U12 = inv(L11) F12, Pb = -L21 inv(L11), Qr = -inv(U11) U12 and F22 - L21 U12.
    Both give the same factor blocks (the stored factor is the same whichever
    kernel produced it)."""
    rng = np.random.default_rng(7)
    for n, m in ((1, 5), (17, 9), (48, 64), (64, 200)):
        F = rng.standard_normal((n + m, n + m)) + 4.0 * (n + m) * np.eye(n + m)
        F11, F12, F21, F22 = F[:n, :n], F[:n, n:], F[n:, :n], F[n:, n:]
        Lw, U = np.eye(n), F11.copy()
        for k in range(n):
            Lw[k + 1:, k] = U[k + 1:, k] / U[k, k]
            U[k + 1:, k:] -= np.outer(Lw[k + 1:, k], U[k, k:])
        U = np.triu(U)
        Li, Ui = np.linalg.inv(Lw), np.linalg.inv(U)
        L21, U12 = F21 @ Ui, Li @ F12
        X = Ui @ Li
        for a, b in ((-L21 @ Li, -F21 @ X), (-Ui @ U12, -X @ F12), (F22 - L21 @ U12, F22 + (-F21 @ X) @ F12)):
            assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(a).max())


def test_one_pass_lu_with_inverses():
    """The pivot steps of the one-CTA fronts (and of the blocked path's
    diagonal blocks), restated: step k publishes row k of A, X, Z and column
    k of A; rows i > k then apply A(i, j) -= l_i A(k, j) (j > k, l_i =
    A(i, k) / A(k, k) stored at j = k), X(i, :) -= l_i X(k, :) and
    Z(i, :) -= A(k, i) Z(k, :) / A(k, k), while row k of Z is scaled by
    1 / A(k, k).  At the end A holds the unit-lower L and U, X = inv(L) and
    Z = inv(U)^T."""
    rng = np.random.default_rng(11)
    for n in (1, 5, 16, 33, 64):
        F = rng.standard_normal((n, n)) + 2.0 * n * np.eye(n)
        A, X, Z = F.copy(), np.eye(n), np.eye(n)
        for k in range(n):
            rp = 1.0 / A[k, k]
            pr, lc, xr, zr = A[k].copy(), A[:, k].copy(), X[k].copy(), Z[k].copy() * rp
            for i in range(k + 1, n):
                l = lc[i] * rp
                A[i, k + 1:] -= l * pr[k + 1:]
                A[i, k] = l
                X[i] -= l * xr
                Z[i] -= pr[i] * zr
            Z[k] = zr
        L, U = np.tril(A, -1) + np.eye(n), np.triu(A)
        assert np.abs(L @ U - F).max() <= 1e-12 * np.abs(F).max()
        assert np.abs(X - np.linalg.inv(L)).max() <= 1e-12
        assert np.abs(Z.T - np.linalg.inv(U)).max() <= 1e-12 * np.abs(np.linalg.inv(U)).max()


def _periodic_matrix(nz, ny, nx, seed=5):
    rng = np.random.default_rng(seed)
    g = synthetic.make_met_bin(rng, nz, ny, nx, terrain_amp=2000.0, rho_profile=True, cmfmc_frac=0.4,
                               periodic=True)
    T = assembly.transport_block(g)
    d = rng.uniform(1e-6, 1e-4, nz * ny * nx)
    return (sp.eye(nz * ny * nx) + 10800.0 * assembly.species_operator(T, d)).tocsr()


@pytest.mark.parametrize("shape,leaf", [((3, 4, 5), 4), ((4, 6, 9), 8), ((3, 9, 4), 6), ((5, 7, 12), 16)])
def test_periodic_ring_dissection_replays_sparse_solve(shape, leaf):
    """A longitude ring is cut by two planes (its first and middle columns);
    the x-neighbours of boxes at columns 0 and nx-1 wrap around.  The replayed
    supernodal factorization and sweeps reproduce scipy's solves with the
    wrap-face couplings in A."""
    from orbit_b200.grid import infer_grid_shape, infer_periodic, stencil_from_matrix
    A = _periodic_matrix(*shape)
    assert infer_grid_shape(A) == shape and infer_periodic(A, shape)
    st = stencil_from_matrix(A, *shape, periodic=True)
    sym = Symbolic(*shape, leaf_cells=leaf, periodic=True)
    n, m, first = sym.array("n"), sym.array("m"), sym.array("first")
    uoff, uidx = sym.array("uoff"), sym.array("uidx")
    assert sorted(sym.array("perm").tolist()) == list(range(sym.N))
    for s in range(len(n)):
        assert np.all(np.diff(uidx[uoff[s]:uoff[s + 1]]) > 0)
        assert np.all(uidx[uoff[s]:uoff[s + 1]] >= first[s] + n[s])
    a, fac = _replay(sym, st)
    rng = np.random.default_rng(2)
    b = rng.standard_normal(sym.N)
    xr = spla.spsolve(A.tocsc(), b)
    assert np.abs(_solve(a, fac, b, trans=False) - xr).max() <= 1e-11 * np.abs(xr).max()
    xtr = spla.spsolve(A.T.tocsc(), b)
    assert np.abs(_solve(a, fac, b, trans=True) - xtr).max() <= 1e-11 * np.abs(xtr).max()


def test_periodic_needs_three_columns():
    with pytest.raises(Exception):
        Symbolic(3, 4, 2, periodic=True)
