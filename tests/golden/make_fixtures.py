"""Regenerate the golden fixtures from the reference's own test cases.

    python tests/golden/make_fixtures.py [REFERENCE_ROOT]

For each of the reference's golden cases (tests/quarter_annular, tests/wetdry,
tests/mass_conservation) this copies the input deck (fort.14, fort.15,
fort.dg) and stores every snapshot of the expected nodal elevation file
fort.63.true as ``expected.npz`` (keys ``it`` and ``eta``, float64 as printed).
These fixtures are what the tests read, so no test needs the reference tree.
"""
from __future__ import annotations

import shutil
import sys
from pathlib import Path

import numpy as np

CASES = ["quarter_annular", "wetdry", "mass_conservation"]
HERE = Path(__file__).resolve().parent


def read_fort63(path: Path):
    lines = [ln for ln in path.read_text().split("\n") if ln.strip()]
    npn = int(lines[1].split()[1])
    its, etas = [], []
    i = 2
    while i < len(lines):
        its.append(int(lines[i].split()[1]))
        etas.append([float(ln.split()[1]) for ln in lines[i + 1:i + 1 + npn]])
        i += 1 + npn
    return np.array(its, np.int64), np.array(etas, np.float64)


def main(ref_root: str = "/root/reference") -> None:
    ref = Path(ref_root) / "tests"
    for case in CASES:
        src, dst = ref / case, HERE / case
        dst.mkdir(exist_ok=True)
        for name in ("fort.14", "fort.15", "fort.dg"):
            shutil.copyfile(src / name, dst / name)
        it, eta = read_fort63(src / "fort.63.true")
        np.savez_compressed(dst / "expected.npz", it=it, eta=eta)
        print(case, eta.shape)


if __name__ == "__main__":
    main(*sys.argv[1:])
