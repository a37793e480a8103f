"""The continuous-batching footprint server: every request's result is the same
alone and in the mix (particle states bit-identical, footprints within float32
atomic-order rounding, 1e-6 relative L1), requests overlap on the device, and the
HBM budget bounds admission."""

from __future__ import annotations

from datetime import timedelta

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _server(syn, grid, **kw):
    from glide_b200.runtime import DomainSpec, EmanuelConfig, FootprintSpec, HannaConfig
    from glide_b200.serving import FootprintServer
    from glide_b200.window import window_from_synthetic

    return FootprintServer(
        grid=grid, met_provider=lambda hk: window_from_synthetic(syn, syn.window_index(hk), grid),
        horizon_start=syn.times[0], horizon_end=syn.times[-1],
        hanna=HannaConfig(meander_enabled=True, max_substeps=6), emanuel=EmanuelConfig(),
        footprint=FootprintSpec((float(syn.lon[0]) - 0.125, float(syn.lon[-1]) + 0.125),
                                (float(syn.lat[0]) - 0.125, float(syn.lat[-1]) + 0.125), len(syn.lon), len(syn.lat),
                                (0.0, 100.0), 1),
        domain=DomainSpec((float(syn.lon[0]), float(syn.lon[-1])), (float(syn.lat[0]), float(syn.lat[-1])), 20000.0),
        device="cuda", keep_footprints=True, **kw)


@pytest.fixture(scope="module")
def met(cuda_device):
    from glide_b200.synthetic import SyntheticMet, SyntheticMetSpec
    from glide_b200.window import grid_from_synthetic

    syn = SyntheticMet(SyntheticMetSpec(nz=30, ny=60, nx=80, lon0=-10.0, lat0=40.0, n_snapshots=10, seed=5),
                       device=cuda_device)
    return syn, grid_from_synthetic(syn).to_device(cuda_device)


def _requests(syn):
    from glide_b200.serving import poisson_requests

    sites = np.array([[0.0, 47.0], [5.0, 50.0], [-4.0, 45.0]])
    return poisson_requests(12, 50.0, sites, syn.times[0] + timedelta(hours=4), 3.0, n_range=(500, 6000),
                            duration_range_h=(1.0, 4.0), seed=11)


def test_result_same_alone_and_in_mix(met):
    syn, grid = met
    reqs = _requests(syn)
    mixed = {r.request_id: r for r in _server(syn, grid, max_active=16, n_streams=8).serve(reqs, realtime=False)}
    assert len(mixed) == len(reqs)
    for req in (reqs[0], reqs[5], reqs[11]):
        alone = _server(syn, grid, max_active=1, n_streams=1).serve([req], realtime=False)[0]
        m = mixed[req.request_id]
        assert alone.n_steps == m.n_steps and alone.escaped == m.escaped
        assert alone.active_particle_steps == m.active_particle_steps
        a, b = alone.footprint.numpy(), m.footprint.numpy()
        assert a.sum() > 0
        assert np.abs(a - b).sum() <= 1e-6 * np.abs(a).sum()


def test_requests_overlap_and_budget_bounds_admission(met):
    syn, grid = met
    reqs = _requests(syn)
    srv = _server(syn, grid, max_active=16, n_streams=8)
    srv.serve(reqs, realtime=False)
    assert srv.stats.peak_active > 1  # several requests in flight at once
    assert srv.stats.completed == len(reqs)
    one = srv.request_bytes(max(reqs, key=lambda r: r.n_particles))
    tight = _server(syn, grid, max_active=16, n_streams=8, hbm_budget_bytes=one)
    res = tight.serve(reqs, realtime=False)
    assert len(res) == len(reqs)
    assert tight.stats.peak_bytes <= one or tight.stats.peak_active == 1


def test_grouped_and_per_stream_servers_agree(met):
    """Grouped launches (one per tick for all requests) and one stream per request give
    the same results."""
    syn, grid = met
    reqs = _requests(syn)
    g = {r.request_id: r for r in _server(syn, grid, max_active=16, grouped=True).serve(reqs, realtime=False)}
    srv = _server(syn, grid, max_active=16, n_streams=8, grouped=False)
    p = {r.request_id: r for r in srv.serve(reqs, realtime=False)}
    assert set(g) == set(p) == {r.request_id for r in reqs}
    for k in g:
        assert g[k].escaped == p[k].escaped and g[k].active_particle_steps == p[k].active_particle_steps
        a, b = g[k].footprint.numpy(), p[k].footprint.numpy()
        assert np.abs(a - b).sum() <= 1e-6 * max(np.abs(a).sum(), 1e-30)


def test_particle_order_does_not_change_results(met):
    """Each request's particles regrouped by work class before every window (the
    default) or stepped in index order: the same results, grouped and per stream."""
    syn, grid = met
    reqs = _requests(syn)
    for grouped in (True, False):
        o = {r.request_id: r for r in _server(syn, grid, max_active=16, grouped=grouped).serve(reqs, realtime=False)}
        i = {r.request_id: r for r in _server(syn, grid, max_active=16, grouped=grouped,
                                              order_particles=False).serve(reqs, realtime=False)}
        assert set(o) == set(i) == {r.request_id for r in reqs}
        for k in o:
            assert o[k].escaped == i[k].escaped and o[k].active_particle_steps == i[k].active_particle_steps
            a, b = o[k].footprint.numpy(), i[k].footprint.numpy()
            assert a.sum() > 0
            assert np.abs(a - b).sum() <= 1e-6 * np.abs(a).sum()



def test_budget_overfilled_with_more_than_a_grouped_launch(met, monkeypatch):
    """60 requests against a budget that holds about 40 of them: admission stops at the
    budget, more than 32 requests are in flight at once, so a tick's grouped launch is
    split (glide_step_batched takes at most 32 batches), and every request's result is
    still the one it has alone."""
    from glide_b200 import serving
    from glide_b200.serving import poisson_requests

    syn, grid = met
    sites = np.array([[0.0, 47.0], [5.0, 50.0], [-4.0, 45.0], [2.0, 43.0]])
    reqs = poisson_requests(60, 1000.0, sites, syn.times[0] + timedelta(hours=4), 3.0, n_range=(300, 3000),
                            duration_range_h=(2.0, 4.0), seed=23)
    probe = _server(syn, grid, max_active=64)
    sizes = sorted((probe.request_bytes(r) for r in reqs), reverse=True)
    budget = float(sum(sizes[:40]))
    groups: list[int] = []
    real = serving.launch_grouped

    def spy(args, stream):
        groups.append(len(args))
        return real(args, stream)

    monkeypatch.setattr(serving, "launch_grouped", spy)
    srv = _server(syn, grid, max_active=64, hbm_budget_bytes=budget)
    res = {r.request_id: r for r in srv.serve(reqs, realtime=False)}
    assert len(res) == len(reqs) and srv.stats.completed == len(reqs)
    assert srv.stats.peak_bytes <= budget
    assert srv.stats.peak_active > 32
    assert max(groups) > 32  # a tick with more batches than one grouped launch holds
    monkeypatch.setattr(serving, "launch_grouped", real)
    for req in (reqs[0], reqs[33], reqs[59]):
        alone = _server(syn, grid, max_active=1).serve([req], realtime=False)[0]
        m = res[req.request_id]
        assert alone.escaped == m.escaped and alone.active_particle_steps == m.active_particle_steps
        a, b = alone.footprint.numpy(), m.footprint.numpy()
        assert np.abs(a - b).sum() <= 1e-6 * max(np.abs(a).sum(), 1e-30)
