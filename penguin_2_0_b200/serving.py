"""Request streams for the serving loop (pg_server_*).

The stream mixes 90% 2D disks drawn as the batched ensemble draws them and
10% 3D disks (nr 64-128, nphi = 3 nr, ntheta 16-32, the same planet, h, alpha
and slope ranges), each for a number of orbits drawn uniformly in a range;
arrivals are a Poisson process.  Grid sizes are drawn from sets whose
azimuthal and radial counts satisfy the reference's chunking rule (no
remainder of 1..5 cells modulo 116)."""
from __future__ import annotations

import math

import numpy as np

from . import ensemble, host
from ._lib import pg_params

SIZES_3D = (64, 80, 96, 112, 128)
NTHETA_3D = (16, 24, 32)


def draw_request(rng: np.random.Generator, index: int, seed: int, orbits_range=(5.0, 50.0),
                 frac_3d: float = 0.1) -> pg_params:
    orbits = rng.uniform(*orbits_range)
    if rng.uniform() < frac_3d:
        nr = int(rng.choice(SIZES_3D))
        nth = int(rng.choice(NTHETA_3D))
        q = 10.0 ** rng.uniform(math.log10(1e-5), math.log10(3e-3))
        h = rng.uniform(0.03, 0.08)
        alpha = 10.0 ** rng.uniform(-4.0, -2.0)
        slope = rng.uniform(0.5, 1.5)
        t_end = orbits * 2.0 * math.pi
        p = host.params(1, imax=nr, jmax=3 * nr, kmax=nth, M_p=q, sc_h=h, ss_alpha=alpha, p_alpha=slope,
                        zmin=math.pi / 2 - 3.0 * h, endtime=t_end, tmovie=t_end, nprin=100)
        p.seed = (seed * 1_000_003 + index) & 0xFFFFFFFFFFFF
    else:
        p = ensemble.draw_disk(rng, index, seed, orbits)
    p.precision = ensemble.precision_for(p)
    return p


def draw_stream(n: int, seed: int = 0, orbits_range=(5.0, 50.0), frac_3d: float = 0.1) -> list[pg_params]:
    rng = np.random.default_rng(seed)
    return [draw_request(rng, i, seed, orbits_range, frac_3d) for i in range(n)]


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed + 7919)
    gaps = rng.exponential(1.0 / rate_per_s, size=n)
    gaps[0] = 0.0
    return np.cumsum(gaps)


def latency_stats(done: list[dict]) -> dict:
    lat = np.array([d["finish_s"] - d["arrival_s"] for d in done])
    wait = np.array([d["admit_s"] - d["arrival_s"] for d in done])
    return dict(p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
                mean_s=float(lat.mean()), max_s=float(lat.max()),
                queue_p50_s=float(np.percentile(wait, 50)), queue_p99_s=float(np.percentile(wait, 99)))
