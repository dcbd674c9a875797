"""Many independent pairs on one or several GPUs: the host side of pair batching.

The reference tracks one pair per `optflow pair` call (rust/crates/optflow-cli/src/run.rs); a batch of
independent pairs of uneven sizes has no exchange step, so it shards across GPUs as replicas: one process
and one engine per GPU, each tracking its share of the pairs, with the results gathered on rank 0 by the
host (torch.distributed object gather; no device collective).

``batch_specs`` draws the uneven batch of seeded pairs (widths and heights independently from
{256, 512, 768, 1024, 1536, 2048}, a random affine strain with |e| <= 0.02, a translation <= 6 px, noise
in [0.003, 0.02]); ``shard`` assigns pairs to ranks by longest-processing-time first on the pixel count,
deterministically, so every rank computes the same plan without communicating; ``run_batch`` tracks one
rank's share and ``gather`` collects every rank's results on rank 0 in the batch's order.
"""
from dataclasses import dataclass

import numpy as np

SIZES = (256, 512, 768, 1024, 1536, 2048)


@dataclass(frozen=True)
class PairSpec:
    index: int
    w: int
    h: int
    exx: float
    eyy: float
    exy: float
    tx: float
    ty: float
    noise: float
    seed: int

    @property
    def pixels(self):
        return self.w * self.h


def batch_specs(n=64, seed=11):
    """The seeded batch of uneven pairs (one PairSpec per pair, in batch order)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        w, h = (int(v) for v in rng.choice(SIZES, 2))
        exx, eyy, exy = rng.uniform(-0.02, 0.02, 3)
        ang = rng.uniform(0, 2 * np.pi)
        t = rng.uniform(0, 6.0)
        noise = rng.uniform(0.003, 0.02)
        out.append(PairSpec(i, w, h, float(exx), float(eyy), float(exy), float(t * np.cos(ang)),
                            float(t * np.sin(ang)), float(noise), int(seed) * 1000 + i))
    return out


def make_pair(spec: PairSpec, engine=None):
    """Renders a spec's pair (uint8-quantised float32 images) and returns (a, b, field)."""
    from . import synth
    p = synth.make_pattern(spec.h, spec.w, seed=spec.seed, rmin=1.5, rmax=2.5)
    field = synth.Field(A=((1 + spec.exx, spec.exy), (spec.exy, 1 + spec.eyy)), c=(spec.w / 2, spec.h / 2),
                        t=(spec.tx, spec.ty))
    a = synth.degrade(synth.render(p, spec.h, spec.w, None, engine=engine), seed=2 * spec.seed,
                      noise=spec.noise, bits=8)
    b = synth.degrade(synth.render(p, spec.h, spec.w, field, engine=engine), seed=2 * spec.seed + 1,
                      noise=spec.noise, bits=8)
    return a, b, field


def shard(specs, world):
    """Pair indices per rank: longest-processing-time first on the pixel count (ties by index), so the
    largest pairs spread first and every rank's load is within one pair of the best split. Deterministic:
    every rank computes the same plan."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0] * world
    plan = [[] for _ in range(world)]
    for s in sorted(specs, key=lambda s: (-s.pixels, s.index)):
        r = min(range(world), key=lambda k: (loads[k], k))
        plan[r].append(s.index)
        loads[r] += s.pixels
    return [sorted(p) for p in plan]


def run_batch(specs, rank, world, track, make=make_pair):
    """Tracks this rank's share of the batch: {index: track(a, b, spec)} for the indices shard() gives
    this rank. ``track`` is the per-pair call (for example a closure over optflow_b200.track_pair)."""
    mine = shard(specs, world)[rank]
    by_index = {s.index: s for s in specs}
    out = {}
    for i in mine:
        a, b, _ = make(by_index[i])
        out[i] = track(a, b, by_index[i])
    return out


def gather(local, rank, world, group=None):
    """Every rank's {index: result} on rank 0, merged in batch order (None on the other ranks).
    With world == 1 it returns the local results sorted."""
    if world == 1:
        return [local[i] for i in sorted(local)]
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        dup = merged.keys() & p.keys()
        if dup:
            raise RuntimeError(f"pairs tracked twice: {sorted(dup)}")
        merged.update(p)
    return [merged[i] for i in sorted(merged)]
