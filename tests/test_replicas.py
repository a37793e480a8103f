"""Release sharding across ranks (the multi-GPU path) on CPU with gloo, world size 2:
each rank runs its share of the releases (here through the oracle, as there is no
GPU), and the merged per-release footprints and escape counts equal those of the
single-process run exactly (particles are independent; releases own disjoint
footprint slices)."""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from glide_b200.replicas import balance_releases, local_release_index, rank_particle_mask

ROOT = Path(__file__).resolve().parents[1]


def test_balance_covers_every_release_once():
    rng = np.random.default_rng(0)
    counts = rng.integers(2000, 20000, 2688)
    for world in (1, 2, 3, 8):
        parts = balance_releases(counts, world)
        allr = np.concatenate(parts)
        assert np.array_equal(np.sort(allr), np.arange(len(counts)))
        loads = np.array([counts[p].sum() for p in parts])
        assert loads.max() - loads.min() <= counts.max()


def test_local_release_index():
    ridx = np.array([0, 0, 3, 5, 3])
    rel = np.array([3, 5])
    m = rank_particle_mask(ridx, rel)
    assert m.tolist() == [False, False, True, True, True]
    assert local_release_index(ridx[m], rel).tolist() == [0, 1, 0]


def _worker(rank: int, world: int, port: int, out_dir: str):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import dataclasses

    import torch.distributed as dist

    from fixtures import load_run, oracle_kwargs
    from glide_b200.replicas import balance_releases, local_release_index, rank_particle_mask, sum_over_ranks
    from oracle.hanna import StepNoise
    from oracle.runtime import run_batch

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    run = load_run("run_small")
    kw = oracle_kwargs(run)
    ridx = run["release_idx"]
    counts = np.bincount(ridx)
    mine = balance_releases(counts, world)[rank]
    m = rank_particle_mask(ridx, mine)
    base_noise = kw["noise_fn"]
    base_unif = kw["conv_uniforms_fn"]
    sel = np.nonzero(m)[0]
    kw.update(particles=kw["particles"][:, m], rel_off=kw["rel_off"][m], win_end_off=kw["win_end_off"][m],
              release_idx=local_release_index(ridx[m], mine),
              grid=dataclasses.replace(kw["grid"], n_releases=len(mine)),
              noise_fn=lambda s: StepNoise(base_noise(s).substep[:, :, sel], base_noise(s).meander[:, sel]),
              conv_uniforms_fn=lambda s: tuple(u[sel] for u in base_unif(s)))
    res = run_batch(**kw, max_steps=40)
    esc = sum_over_ranks(int(sum(res.escaped_per_step)))
    np.savez(Path(out_dir) / f"rank{rank}.npz", releases=mine, footprint=res.footprint, esc_total=esc,
             particles=res.particles, sel=sel)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_matches_single_process(tmp_path):
    from fixtures import load_run, oracle_kwargs
    from oracle.runtime import run_batch

    port = 29500 + (os.getpid() % 1000)
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    run = load_run("run_small")
    full = run_batch(**oracle_kwargs(run), max_steps=40)
    merged = np.zeros_like(full.footprint)
    parts = np.zeros_like(full.particles)
    for rank in (0, 1):
        z = np.load(tmp_path / f"rank{rank}.npz")
        merged[z["releases"]] = z["footprint"]
        parts[:, z["sel"]] = z["particles"]
        assert int(z["esc_total"]) == sum(full.escaped_per_step)
    np.testing.assert_array_equal(merged, full.footprint)
    np.testing.assert_array_equal(parts, full.particles)
