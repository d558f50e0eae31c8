"""Copy the reference's own 2-D FP64 golden fixtures for this path.

finitevolX ships golden outputs under ``tests/fixtures/golden`` (18x18
arrays, produced by its ``tests/fixtures/_gen_golden.py`` with
``jax_enable_x64``).  The files used to pin the oracle are copied verbatim
into ``tests/golden/ref`` so the tests do not need the reference tree at run
time.  Run from the repository root:

    python tests/golden/import_reference_goldens.py /path/to/finitevolX
"""

import pathlib
import shutil
import sys

PREFIXES = (
    "Advection2D____call___",
    "Difference2D__",
    "Interpolation2D__",
    "Diffusion2D__",
    "BiharmonicDiffusion2D__",
    "Divergence2D__",
    "Coriolis2D__",
    "Vorticity2D__",
    "MomentumAdvection2D__",
)


def main(ref_root: str) -> int:
    src = pathlib.Path(ref_root) / "tests" / "fixtures" / "golden"
    dst = pathlib.Path(__file__).resolve().parent / "ref"
    dst.mkdir(exist_ok=True)
    n = 0
    for f in sorted(src.glob("*.npz")):
        if f.name.startswith(PREFIXES):
            shutil.copyfile(f, dst / f.name)
            n += 1
    print(f"copied {n} golden files to {dst}")
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/import_reference_goldens.py /path/to/finitevolX")
    sys.exit(main(sys.argv[1]))
