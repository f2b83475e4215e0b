"""Generate the golden near-field vectors from the reference's own CPU kernel.

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


def main():
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
