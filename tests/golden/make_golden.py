"""Generate the golden near-field vectors from the reference's own CPU kernel,
and the golden kick vectors from the reference's own kick.

    python tests/golden/make_golden.py

Runs singlestep/Direct/direct.cpp (Direct::Execute + directkernel<0>),
compiled unmodified from the reference sources into
oracle/_ref/libnfref_<softening>_strict.so (oracle/Makefile, -O2
-ffp-contract=off), driven by the ExecuteSlabCPU cell loop of
oracle/ref_shim.cpp, on small seeded boxes, and stores inputs and outputs as
.npz fixtures next to this script.  The fixtures travel with the repository;
the reference sources do not need to be present to use them.
"""
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))

import importlib.util  # noqa: E402

spec = importlib.util.spec_from_file_location(
    "abacus_public_b200", ROOT / "abacus-public_b200" / "__init__.py",
    submodule_search_locations=[str(ROOT / "abacus-public_b200")])
mod = importlib.util.module_from_spec(spec)
sys.modules["abacus_public_b200"] = mod
spec.loader.exec_module(mod)
from abacus_public_b200 import synth  # noqa: E402

import oracle as O  # noqa: E402

CASES = [
    # name, box factory, n_side (softening spacing), slabs
    ("uniform_cpd7", lambda: synth.uniform_box(3000, 7, seed=11), 14, [0, 3, 6]),
    ("clustered_cpd9", lambda: synth.clustered_box(6000, 9, seed=12, n_clumps=6), 18, [0, 4, 8]),
    ("sparse_cpd5", lambda: synth.uniform_box(300, 5, seed=13), 7, [0, 2, 4]),
]


# RescaleAndCoAddAcceleration + KickSlab (singlestep/Timestep/kick.cpp,
# compiled unmodified into oracle/_ref/libnfref_kick_<softening>.so with the
# density channel on) on seeded arrays: two slabs of cpd 5, up to 40
# particles per cell, near accelerations with a density w, far accelerations
# and velocities.
KICK = dict(cpd=5, omega_m=0.3089, omega_smooth=0.0, np_total=256 ** 3, make_glass=0,
            kick1=0.0131, kick2=0.0117, b2=2.5e-7)


def kick_main():
    for soft, sli in ((0, 1.0 / 256 / 40), (1, 2.15517 / 256 / 40)):
        rng = np.random.default_rng(20 + soft)
        cpd = KICK["cpd"]
        counts = rng.integers(0, 41, size=2 * cpd * cpd)
        n = int(counts.sum())
        scale = 1e11 if soft == 1 else 1e4  # raw near output: single spline lacks eps^-3
        nacc = np.zeros((n, 4), np.float32)
        nacc[:, :3] = rng.standard_normal((n, 3)) / scale * 1e7
        nacc[:, 3] = KICK["b2"] * (1 + 20 * rng.random(n))
        far = (rng.standard_normal((n, 3)) * 1e7).astype(np.float32)
        vel = (rng.standard_normal((n, 3)) * 1e-2).astype(np.float32)
        acc, v, stats, dens = O.ref_rescale_and_kick(
            soft, nacc, far, vel, counts, cpd, KICK["omega_m"], KICK["omega_smooth"],
            KICK["np_total"], KICK["make_glass"], sli, np.float32(KICK["kick1"]),
            np.float32(KICK["kick2"]), np.float32(KICK["b2"]))
        out = HERE / f"kick_{O.SOFTENING_NAMES[soft]}.npz"
        np.savez_compressed(out, softening=soft, cpd=cpd, counts=counts, nacc=nacc, far=far,
                            vel=vel, softening_length_internal=sli,
                            **{k: v_ for k, v_ in KICK.items() if k != "cpd"},
                            acc_out=acc, vel_out=v, stats_out=stats, dens_out=dens)
        print(out.name, n, "particles")


def main():
    kick_main()
    for name, mk, nside, slabs in CASES:
        box = mk()
        for soft in range(4):
            eps = synth.kernel_eps(soft, synth.plummer_eps(nside))
            acc = np.zeros((box.n, 3), dtype=np.float32)
            for s in slabs:
                O.ref_slab(box, soft, eps, s, flavour="strict", acc=acc)
            rows = np.concatenate([np.arange(*box.slab_range(s)) for s in slabs])
            out = HERE / f"{name}_{O.SOFTENING_NAMES[soft]}.npz"
            np.savez_compressed(out, cpd=box.cpd, x=box.x, y=box.y, z=box.z,
                                cell_start=box.cell_start, softening=soft,
                                eps=np.float32(eps), slabs=np.array(slabs), rows=rows,
                                acc=acc[rows])
            print(out.name, box.n, "particles", rows.size, "sinks")


if __name__ == "__main__":
    main()
