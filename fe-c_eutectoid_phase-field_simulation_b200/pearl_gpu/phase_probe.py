"""Run single phases of the hot path as their own launches, for profiling one
phase at a time (the time step itself is one persistent kernel, so a profiler
sees all phases as one launch).

    python -m pearl_gpu.phase_probe propose   --nx 2048 --ny 4096 --repeat 3
    python -m pearl_gpu.phase_probe diffusion --nx 2048 --ny 4096 --repeat 3

`propose` launches propose_phi (plus the mixture of the trial phi) on the large
FP64 workload; `diffusion` launches the implicit solve (set-up, PCG, final)
on the trial phase fields of one proposal."""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))


def main(argv=None) -> int:
    import pearl_gpu
    from pearl_gpu import workloads

    ap = argparse.ArgumentParser()
    ap.add_argument("phase", choices=["propose", "diffusion"])
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=4096)
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args(argv)
    w = workloads.plain_large(nx=args.nx, ny=args.ny, pairs=max(1, args.nx // 32))
    dt = w.meta["dt"]
    with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        for _ in range(args.repeat):
            if args.phase == "propose":
                change = ctx.propose_phi(dt)
                print(f"propose: max change {change:.3e}, {ctx.stats()['last_ms']:.3f} ms")
            else:
                ctx.propose_phi(dt)
                d = ctx.implicit_diffusion(dt)
                print(f"diffusion: ok {d['ok']}, {d['it']} CG iterations, {ctx.stats()['last_ms']:.3f} ms")
    return 0


if __name__ == "__main__":
    sys.exit(main())
