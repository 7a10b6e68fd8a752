"""Autotuner of the tile kernels.

For one (n, nst, K) it times, with the library's phase events, the energy
tiles over (ket-chunk width LC_e, register variant minb_e) and the gradient
tiles over (LC_g, minb_g) -- the two are independent -- and keeps the fastest
of each.  Results are cached in a JSON file keyed by GPU name, n, nst and a K
bucket (powers of two), so a run pays for tuning once.

The search space:
  LC_e   ket chunk of an energy tile (kets per warp per tile)
  LC_g   ket chunk of a gradient tile (also sets the partial-buffer depth)
  minw   minimum resident warps per SM the kernel is compiled for (one warp
         per block): 8 -> up to 255 registers per thread, 12 -> 168, 16 -> 128,
         20 -> 96 (the register file is split between the four schedulers, so
         these are the only distinct budgets)
  sym    gradient pass over unordered pairs (bra and ket gradient per term,
         when the symmetry set is closed under inverse) instead of ordered
         pairs, with its own ket chunk lc_s and variant minw_s; sym = 2 fuses
         it with the energy pass (one pass for H, S and both gradients), kept
         when its total beats the best separate energy + gradient passes
  npc    splits of the symmetry terms per tile of the fused pass (one-warp
         variants): tried when the basis has few tiles (SPLIT_TILES), where each
         tile's chain of LC x nst terms, not the GPU's width, sets the time
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import torch

from . import _lib
from .engine import Engine

CACHE = os.environ.get("NECG_TUNE_CACHE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "tune_cache.json"))

LC_E = (2, 4, 8, 16, 32)
LC_G = (4, 8, 16, 32, 64)
MINB = (8, 12, 16, 20)
MINB_GRAD_EXTRA = (112, 116)  # gradient kernel with shared-memory accumulators
LC_S = (1, 2, 4, 8, 16)       # kets per tile of the symmetric gradient pass
MINW_SYM = (8, 12)
MINW_FUSED = (8, 12, 16, 108, 112, 118, 122, 208, 218, 228, 222, 232, 248, 258, 268)
SPLITS = (1, 2, 3, 4, 6, 8, 12, 24)
SPLIT_TILES = 2048  # try splits below this many fused tiles
# 100 + w: ket records re-read at each use (118 / 122: staged in shared memory,
# 8 / 12 warps); 2xy: lockstep blocks (208 8 warps,
# 218 + bras in shared memory, 228 + ket records in shared memory, 248 as 228
# without a barrier per term, 258 / 268 as 228 with half the warps taking their
# per-term barrier inside the term, 222 / 232 as 218 / 228 with 12 warps); a
# variant whose shared memory does not fit for n is refused by
# necg_set_symmetric and skipped


def fused_tiles(K: int, lc: int) -> int:
    """Tiles (32-row block, chunk of lc kets) over the lower triangle of K."""
    return sum(min(kb * 32 + 31, K - 1) // lc + 1 for kb in range((K + 31) // 32))


def _bucket(K: int) -> int:
    b = 16
    while b < K:
        b *= 2
    return b


def _key(n: int, nst: int, K: int) -> str:
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return f"{name}|n{n}|nst{nst}|K{_bucket(K)}"


def load_cache() -> dict:
    try:
        with open(CACHE) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict) -> None:
    tmp = f"{CACHE}.{os.getpid()}.tmp"  # ranks of one node may save at the same time
    with open(tmp, "w") as fh:
        json.dump(cache, fh, indent=1, sort_keys=True)
    os.replace(tmp, CACHE)


def _phase_times(eng: Engine, x: torch.Tensor, K: int, reps: int) -> np.ndarray:
    L = eng.L
    g = torch.empty_like(x)
    f = torch.empty(1, dtype=torch.float64, device=x.device)
    buf = (ctypes.c_double * 5)()
    out = []
    for _ in range(reps):
        _lib.check(L.necg_outprod(eng.h, K, x.data_ptr(), f.data_ptr(), g.data_ptr(), None, None,
                                  torch.cuda.current_stream().cuda_stream), "necg_outprod")
        _lib.check(L.necg_phase_ms(eng.h, buf), "necg_phase_ms")
        out.append(list(buf))
    return np.array(out)


def tune(eng: Engine, x, K: int, reps: int = 3, report: bool = False) -> dict:
    """Time every candidate on this engine and input; returns the best setting."""
    L = eng.L
    x = eng._tensor(x)
    _lib.check(L.necg_profile(eng.h, 1), "necg_profile")
    L.necg_set_symmetric(eng.h, 0, 4, 8)
    rows = []
    best_e = (float("inf"), None)
    best_g = (float("inf"), None)
    for minb in MINB + MINB_GRAD_EXTRA:
        for lc_e, lc_g in zip(LC_E, LC_G):
            _lib.check(L.necg_set_tiles(eng.h, lc_e, lc_g), "necg_set_tiles")
            _lib.check(L.necg_set_variant(eng.h, minb if minb < 100 else 8, minb), "necg_set_variant")
            _phase_times(eng, x, K, 1)  # warm-up (also builds the energy tile list)
            t = _phase_times(eng, x, K, reps).min(axis=0)
            e_ms, g_ms = float(t[1]), float(t[3] + t[4])
            rows.append({"minb": minb, "lc_e": lc_e, "lc_g": lc_g, "energy_ms": e_ms, "grad_ms": g_ms})
            if e_ms < best_e[0] and minb < 100:
                best_e = (e_ms, (lc_e, minb))
            if g_ms < best_g[0]:
                best_g = (g_ms, (lc_g, minb))
    res = {"lc_e": best_e[1][0], "minb_e": best_e[1][1], "lc_g": best_g[1][0], "minb_g": best_g[1][1],
           "energy_ms": best_e[0], "grad_ms": best_g[0], "sym": 0, "lc_s": 4, "minw_s": 8}
    # the symmetric gradient pass (unordered pairs), when the symmetry set allows it
    if L.necg_set_symmetric(eng.h, 1, 4, 8) == _lib.NECG_OK:
        _lib.check(L.necg_set_tiles(eng.h, res["lc_e"], res["lc_g"]), "necg_set_tiles")
        _lib.check(L.necg_set_variant(eng.h, res["minb_e"], res["minb_g"]), "necg_set_variant")
        for minw in MINW_SYM:
            for lc in LC_S:
                _lib.check(L.necg_set_symmetric(eng.h, 1, lc, minw), "necg_set_symmetric")
                _phase_times(eng, x, K, 1)
                t = _phase_times(eng, x, K, reps).min(axis=0)
                g_ms = float(t[3] + t[4])
                rows.append({"sym": 1, "minw": minw, "lc_s": lc, "grad_ms": g_ms})
                if g_ms < res["grad_ms"]:
                    res.update(grad_ms=g_ms, sym=1, lc_s=lc, minw_s=minw)
        # fused energy + symmetric gradient pass: phase 1 is the whole pair pass
        best_sep = res["energy_ms"] + res["grad_ms"]
        fused = None
        for minw in MINW_FUSED:
            for lc in LC_S:
                if L.necg_set_symmetric(eng.h, 2, lc, minw) != _lib.NECG_OK:
                    continue
                splits = [1]
                if minw < 200 and fused_tiles(K, lc) < SPLIT_TILES:
                    splits = [s for s in SPLITS if s <= eng.nst]
                for npc in splits:
                    _lib.check(L.necg_set_splits(eng.h, npc), "necg_set_splits")
                    _phase_times(eng, x, K, 1)
                    t = _phase_times(eng, x, K, reps).min(axis=0)
                    tot = float(t[1] + t[3] + t[4])
                    rows.append({"sym": 2, "minw": minw, "lc_s": lc, "npc": npc, "total_ms": tot})
                    if tot < best_sep and (fused is None or tot < fused[0]):
                        fused = (tot, lc, minw, npc)
                L.necg_set_splits(eng.h, 1)
        if fused is not None:
            res.update(sym=2, lc_s=fused[1], minw_s=fused[2], npc=fused[3], fused_ms=fused[0])
    if report:
        res["table"] = rows
    apply(eng, res)
    return res


def apply(eng: Engine, cfg: dict) -> None:
    _lib.check(eng.L.necg_set_tiles(eng.h, int(cfg["lc_e"]), int(cfg["lc_g"])), "necg_set_tiles")
    _lib.check(eng.L.necg_set_variant(eng.h, int(cfg["minb_e"]), int(cfg["minb_g"])), "necg_set_variant")
    sym = int(cfg.get("sym", 0))
    rc = eng.L.necg_set_symmetric(eng.h, sym, int(cfg.get("lc_s", 4)), int(cfg.get("minw_s", 8)))
    if rc != _lib.NECG_OK and sym:
        _lib.check(rc, "necg_set_symmetric")
    _lib.check(eng.L.necg_set_splits(eng.h, min(int(cfg.get("npc", 1)), eng.nst)), "necg_set_splits")


def tuned(eng: Engine, x, K: int, retune: bool = False) -> dict:
    """Apply the cached setting for (GPU, n, nst, K bucket), tuning on a miss."""
    cache = load_cache()
    key = _key(eng.n, eng.nst, K)
    if key in cache and not retune:
        apply(eng, cache[key])
        return cache[key]
    res = tune(eng, x, K)
    cache[key] = {k: v for k, v in res.items() if k != "table"}
    try:
        save_cache(cache)
    except OSError:
        pass
    return cache[key]
