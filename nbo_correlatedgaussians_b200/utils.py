"""Drop-in utilities (python/utils.py:26-106): biout, get_current_time, vech,
tab, and the Boys function f0/df0 evaluated by the CUDA library."""
from __future__ import annotations

from datetime import datetime, timezone

import numpy as np

_OUTPUT_FILE = "necg.out"


def biout(string: str) -> None:
    """Print and append to necg.out (python/utils.py:26-30)."""
    print(string)
    with open(_OUTPUT_FILE, "a", encoding="utf-8") as fh:
        fh.write(string + "\n")


def get_current_time() -> tuple[str, str, str]:
    now = datetime.now(tz=timezone.utc)
    return now.strftime("%Y%m%d"), now.strftime("%H%M%S") + ".000", "+0000"


def vech(Ma: np.ndarray, dim: int) -> np.ndarray:
    """Lower triangle, column by column (python/utils.py:42-55)."""
    Ma = np.asarray(Ma)
    rows, cols = np.tril_indices(dim)
    order = np.lexsort((rows, cols))  # column-major
    return Ma[rows[order], cols[order]].astype(np.float64)


def tab(ax: np.ndarray, n: int, m: int) -> None:
    """Print ax (n x m) in blocks of ten columns (python/utils.py:58-75)."""
    for j0 in range(0, m, 10):
        j1 = min(j0 + 10, m)
        print("      " + "".join(f"{j + 1:24d}" for j in range(j0, j1)))
        for i in range(n):
            print(f"{i + 1:3d}   " + "".join(f"{ax[i, j]:23.15f}" for j in range(j0, j1)))


def f0(z: float) -> float:
    """Boys function F0 by the reference's Pade form, evaluated on the GPU."""
    from .engine import boys_f0
    return float(boys_f0(z)[0][0])


def df0(z: float) -> float:
    """Derivative of f0, evaluated on the GPU."""
    from .engine import boys_f0
    return float(boys_f0(z)[1][0])
