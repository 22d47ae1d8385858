"""Every kernel of the step, launched once each, for per-kernel profiler captures.

    python -m retainwall_code_b200.profiling [--nx 100] [--steps 1] [--vx 0.05]

Creates the retaining-wall case with a soil block of nx x 80 x 120 particles
(nx = 100: 0.96M soil particles; the context's own first neighbour search sorts the
particles, so the cell-list kernels run on real work), turns the step graph's
conditional gates off, and runs `steps` whole steps as per-stage calls (the kernels of
each stage launched directly on the context's stream), then the Shepard filter stage
and both wall resultants.  With --vx the soil starts moving along +x at that speed
(m/s), its block moved by dx/10 along x first: the generator's lattice keeps every
particle at least 0.05 dx from every cell face, and the shift brings a band of
particles up to the x faces.  At 0.05 m/s about 150 particles change cell in the first
step, so the second step's predictor section updates the candidate lists after a sort
(mark dilation, list carry, rebuilds next to the marked cells), as the long run does
once the wall has moved the soil."""
from __future__ import annotations

import argparse

from . import LoquatSph, _abi, cases


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=100)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--vx", type=float, default=0.0)
    args = ap.parse_args()
    case = cases.retaining_wall(nx=args.nx)
    if args.vx:
        case.pospres[case.npb:, 0] += 0.1 * case.params["dr"]
        case.velrhop[case.npb:, 0] = args.vx
    sim = LoquatSph(case=case)
    sim.set_option(_abi.OPT_GRAPH_GATES, 0)
    for _ in range(args.steps):
        sim.step_calculation()
        sim.predictor_section()
        sim.corrector_section()
        sim.end_step()
    sim.stress_regularization()
    f0, f1 = sim.wall_force(0), sim.wall_force(1)
    sim.synchronize()
    inf = sim.info()
    print(f"steps {inf.step}; wall resultant {f0[0]:.6g} N (nearest wall), {f1[0]:.6g} N (strip); "
          f"sorted sections {inf.n_sorts}, list updates {inf.n_list_updates} ({inf.n_lists_rebuilt} lists rebuilt)")


if __name__ == "__main__":
    main()
