"""Golden vectors produced by the reference's own CPU code (see make_golden.py)."""
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def load(name: str) -> dict:
    with np.load(HERE / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def names(prefix: str = "") -> list[str]:
    return sorted(p.stem for p in HERE.glob(f"{prefix}*.npz"))
