"""Per-(nx, nv)-bucket tuning of the implicit step kernel's tile height.

The step kernel processes tiles of 32 velocities x R scan positions (R in
{8, 16, 24, 32}).  Short tiles give small instances more tiles (more
parallelism, shorter per-tile latency); tall tiles amortise the look-back and
the row-block bookkeeping on large instances.  ``tune`` times each candidate
R on up to ``per_bucket`` instances of every bucket (one plan per candidate,
a warm-up step, then timed steps with CUDA events) and keeps the fastest.
The table maps bucket names (``batch.bucket_of``) to R and is saved as
JSON; ``BatchSolver`` and the serving loop read it.  Results depend on R at
rounding level only.
"""
from __future__ import annotations

import json
from collections import defaultdict
from pathlib import Path
from typing import Sequence

import torch

from .batch import InstanceDesc, bucket_of, make_state, spec_of
from .plan import ImplicitPlan, implicit_params_struct

DEFAULT_TABLE = Path(__file__).resolve().parent / "tune_table.json"
CANDIDATES = (8, 16, 32)


def _time_plan(descs, R, params, steps):
    states = [make_state(d) for d in descs]
    specs = [spec_of(d, s) for d, s in zip(descs, states)]
    plan = ImplicitPlan(specs, implicit_params_struct(None, tile_rows=R, **params))
    plan.step(1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    plan.step(steps)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def tune(descs: Sequence[InstanceDesc], params: dict | None = None, candidates=CANDIDATES,
         per_bucket: int = 8, steps: int = 4) -> dict:
    params = params or dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16)
    groups = defaultdict(list)
    for d in descs:
        groups[bucket_of(d.nx, d.nv)].append(d)
    table, timings = {}, {}
    for b, ds in sorted(groups.items()):
        sample = ds[:per_bucket]
        ms = {R: _time_plan(sample, R, params, steps) for R in candidates}
        table[b] = min(ms, key=ms.get)
        timings[b] = {str(R): round(t, 4) for R, t in ms.items()}
    return {"table": table, "ms_per_step": timings, "candidates": list(candidates),
            "per_bucket": per_bucket, "steps": steps}


def save(result: dict, path=DEFAULT_TABLE) -> None:
    Path(path).write_text(json.dumps(result, indent=1, sort_keys=True))


def load(path=DEFAULT_TABLE) -> dict | None:
    p = Path(path)
    if not p.exists():
        return None
    return json.loads(p.read_text()).get("table")


if __name__ == "__main__":
    import sys

    from .batch import sample_instances

    res = tune(sample_instances(256, seed=0))
    save(res, sys.argv[1] if len(sys.argv) > 1 else DEFAULT_TABLE)
    print(json.dumps(res["table"], indent=1))
