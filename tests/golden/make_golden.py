"""Generate the golden fixtures from the REFERENCE's own step functions.

Runs oracle/_ref/dnsref (the reference's DNS-solver/src files compiled
unmodified against the single-rank MPI stand-in) on small seeded inputs and
stores inputs, final states, per-step force/density and the parsed text logs
(energy.txt, flowrate.txt, massrate.txt, str-up.txt, str-do.txt, w-str.txt,
p-grad.txt) and statistics (turb-fld) / vel / den outputs as npz files.

    python tests/golden/make_golden.py [step] [quadrant] [correl]
        (needs the reference sources at $REF_SRC; run once; no argument: all)

The quadrant and correlation fixtures hold the reference post-processing
functions' outputs on the velocity field of a channel stepped by the oracle;
the field itself is regenerated from the stored seed by the tests.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "dns-solvers_b200"))
import inputs  # noqa: E402
import oracle  # noqa: E402

# name, (nx, ny, nz), texture (reference function), const_g, omega, steps, seed
CASES = [
    ("smooth_g_9x5x7", (9, 5, 7), "smooth", True, 1.5, 24, 1),
    ("smooth_q_12x8x6", (12, 8, 6), "smooth", False, 1.9, 21, 2),
    ("ridges_g_16x8x6", (16, 8, 6), "ridges", True, 1.2, 20, 3),
    ("ridges_q_8x12x5", (8, 12, 5), "ridges", False, 1.7, 17, 4),
    ("posts_g_8x8x6", (8, 8, 6), "posts", True, 1.9, 18, 5),
    ("posts_q_12x8x5", (12, 8, 5), "posts", False, 1.4, 15, 6),
]


# quadrant-analysis cases: name, (nx, ny, nz), steps of the oracle, seed
QUADRANT_CASES = [
    ("quadrant_16x12x10", (16, 12, 10), 9, 11),
    ("quadrant_33x20x14", (33, 20, 14), 6, 12),
]


# two-point correlation cases (2pt-correlations/src: ycorrel.c, xcorrel.c):
# name, (nx, ny, nz), steps of the oracle, seed; nx is the program's
# compile-time streamwise size
CORREL_CASES = [
    ("correl_512x12x8", (512, 12, 8), 5, 21),
    ("correl_512x9x7", (512, 9, 7), 4, 22),
]


def correl_field(nx, ny, nz, steps, seed):
    st = inputs.laminar_state(nx, ny, nz, 0.08, 0.3, seed)
    oracle.run(st, inputs.flags_smooth(nx, ny, nz), 1.7, gx=2e-5, const_g=True, nsteps=steps)
    return oracle.moments(st)[0]


def case_input(nx, ny, nz, seed):
    # perturbed Poiseuille at equilibrium, +-10% of u_max on every component
    return inputs.laminar_state(nx, ny, nz, 0.08, 0.1, seed)


def main():
    which = set(sys.argv[1:]) or {"step", "quadrant", "correl"}
    oracle.build()
    for name, (nx, ny, nz), tex, cg, om, steps, seed in CASES if "step" in which else []:
        s0 = case_input(nx, ny, nz, seed)
        r = oracle.run_reference(s0, om, ubulk=0.06, gx=2e-5, const_g=cg, nsteps=steps, texture=tex,
                                 stats_every=steps - 1, vel_every=steps - 1)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            dims=np.array([nx, ny, nz]), texture=tex, const_g=cg, omega=om, ubulk=0.06, gx=2e-5, steps=steps,
            seed=seed, state=r["state"], force=r["force"], rho=r["rho"],
            logs=np.stack([r[n] for n in ("energy", "flowrate", "massrate", "stup", "stdown", "stress", "pgrad")], 1),
            stats_first=r["stats"][0], stats_last=r["stats"][-1], vel_last=r["vel"][-1], den_last=r["den"][-1])
        print(name, "ok")
    # quadrant analysis (quadrant-analysis/src/qUADrantA.c) of the velocity
    # field of a stepped channel, through the reference's own function
    for name, (nx, ny, nz), steps, seed in QUADRANT_CASES if "quadrant" in which else []:
        st = inputs.laminar_state(nx, ny, nz, 0.08, 0.3, seed)
        oracle.run(st, inputs.flags_smooth(nx, ny, nz), 1.7, gx=2e-5, const_g=True, nsteps=steps)
        vel, _ = oracle.moments(st)
        q, dq, uw = oracle.quadrant_reference(vel, label=7)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), dims=np.array([nx, ny, nz]), steps=steps,
                            seed=seed, quadrant=q, dquadrant=dq, uw=uw)
        print(name, "ok")
    # two-point correlations: the restated mean subtraction (the program's own
    # cannot run as shipped), then the reference's ycorrel and xcorrel
    for name, (nx, ny, nz), steps, seed in CORREL_CASES if "correl" in which else []:
        fl, _ = oracle.mean_subtract(correl_field(nx, ny, nz, steps, seed))
        xc, yc = oracle.correlations_reference(fl, label=3)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), dims=np.array([nx, ny, nz]), steps=steps,
                            seed=seed, xcorl=xc, ycorl=yc)
        print(name, "ok")


if __name__ == "__main__":
    main()
