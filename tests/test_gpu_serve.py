"""Serving loop: every request's result is the same alone and in the mix."""
import numpy as np
import pytest

from oracle import assembly, orbit as oorbit

pytestmark = pytest.mark.gpu


def _provider_and_species():
    from orbit_b200 import synthetic
    cache = {}

    def species_of(domain, month):
        key = (domain, month)
        if key not in cache:
            nz, ny, nx = domain
            mets = synthetic.make_met(100 + 31 * month + nx, nz, ny, nx, cmfmc_frac=0.3)
            spc = [synthetic.make_species(200 + s, nz, ny, nx) for s in range(3)]
            cache[key] = (mets, spc)
        return cache[key]

    def provider(domain, month):
        mets, spc = species_of(domain, month)
        return mets, [s.sink_diag(mets) for s in spc]

    return provider, species_of


def _requests(species_of):
    from orbit_b200.serve import OrbitRequest
    rng = np.random.default_rng(4)
    out = []
    for q in range(9):
        domain = [(5, 8, 9), (6, 10, 12)][q % 2]
        month = q % 3 % 2
        kind = ["forward", "marginal", "adjoint"][q % 3]
        sp = [q % 3] if q % 2 else [0, 2]
        mets, spc = species_of(domain, month)
        N = domain[0] * domain[1] * domain[2]
        if kind == "adjoint":
            F = np.stack([rng.random((8, N)) for _ in sp])
        else:
            F = np.stack([spc[s].emis * (1.0 + (0.2 if kind == "marginal" else 0.0)) for s in sp])
        out.append(OrbitRequest(domain=domain, month=month, kind=kind, species=sp, forcing=F, tol=1e-10))
    return out


def test_results_same_alone_and_in_the_mix():
    from orbit_b200.serve import OrbitServer
    provider, species_of = _provider_and_species()
    mix = _requests(species_of)
    srv = OrbitServer(provider, hbm_budget_bytes=4e9, slots=4, precision=32, workers=2).start()
    for r in mix:
        srv.submit(r)
    for r in mix:
        assert r.done.wait(120)
    srv.stop()
    assert all(r.error is None for r in mix), [r.error for r in mix]
    assert srv.batches < len(mix)  # requests were batched together
    alone = _requests(species_of)
    for r in alone:
        s1 = OrbitServer(provider, hbm_budget_bytes=4e9, slots=4, precision=32, workers=1).start()
        s1.submit(r)
        assert r.done.wait(120)
        s1.stop()
    for a, b in zip(mix, alone):
        scale = np.abs(b.result).max()
        assert np.abs(a.result - b.result).max() <= 1e-10 * scale
    # one forward request against the oracle (mixed precision within 1e-6)
    r = next(x for x in mix if x.kind == "forward")
    mets, spc = species_of(r.domain, r.month)
    s = r.species[0]
    d = spc[s].sink_diag(mets)
    lus = [oorbit.factor_one_bin(assembly.species_operator(assembly.transport_block(g), d[t]))
           for t, g in enumerate(mets)]
    ref, _ = oorbit.solve_orbit_one_species(lus, list(r.forcing[0]), tol=1e-12)
    ref = np.stack(ref)
    assert np.abs(r.result[0] - ref).max() <= 1e-6 * np.abs(ref).max()


def test_full_domain_requests_same_alone_and_in_the_mix():
    """80x72x15 (86,400 cells): a forward request and a marginal request
    (emission perturbations of 5x5 surface patches solved on the same species'
    operator) arriving together are batched; each equals its solve alone."""
    from orbit_b200.serve import OrbitRequest, OrbitServer
    provider, species_of = _provider_and_species()
    domain, month = (15, 72, 80), 0
    mets, spc = species_of(domain, month)
    nz, ny, nx = domain
    N = nz * ny * nx

    def reqs():
        fwd = OrbitRequest(domain=domain, month=month, kind="forward", species=[0, 1],
                           forcing=np.stack([spc[0].emis, spc[1].emis]), tol=1e-8)
        F = np.zeros((3, 8, nz, ny, nx))
        e0 = spc[1].emis.reshape(8, nz, ny, nx)
        for q, (j0, i0) in enumerate([(3, 4), (30, 40), (60, 70)]):
            F[q, :, 0, j0:j0 + 5, i0:i0 + 5] = 0.1 * e0[:, 0, j0:j0 + 5, i0:i0 + 5]
        mar = OrbitRequest(domain=domain, month=month, kind="marginal", species=[1, 1, 1],
                           forcing=F.reshape(3, 8, N), tol=1e-8)
        return [fwd, mar]

    mix = reqs()
    srv = OrbitServer(provider, hbm_budget_bytes=60e9, slots=8, precision=32, workers=2).start()
    for r in mix:
        srv.submit(r)
    for r in mix:
        assert r.done.wait(300)
    srv.stop()
    assert all(r.error is None for r in mix), [r.error for r in mix]
    assert srv.batches <= 2  # same entry and direction: batched unless the first started alone
    for a in mix:
        (b,) = [x for x in reqs() if x.kind == a.kind]
        s1 = OrbitServer(provider, hbm_budget_bytes=60e9, slots=8, precision=32, workers=1).start()
        s1.submit(b)
        assert b.done.wait(300)
        s1.stop()
        assert np.all(a.info[:, 4] > 0) and np.all(b.info[:, 4] > 0)
        scale = np.abs(b.result).max()
        assert np.abs(a.result - b.result).max() <= 1e-6 * scale
