"""The persisted autotune table of the 2D stage kernels' tile variants.

``GpuSolve.autotune`` times every tile variant of a solve on its own state;
the library remembers the winner per key (P, flux, dissipation form,
geometry) for the whole process.  Solves created afterwards start from their
key's variant, and the batched engine runs each group of instances with it.
``save``/``load`` persist the table as JSON; ``frforge_b200/autotune_b200.json``
is the table measured on a B200 and is what ``load_default`` reads.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _lib as L

AV = {"none": 0, "br0": 1, "local_dd": 2}
DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_b200.json")


def key_of(p: int, flux: str, av: str, curved: bool):
    return int(p), L.FLUX[flux], AV[av], 1 if curved else 0


def set_variant(p: int, flux: str, av: str, curved: bool, variant: int) -> None:
    L.check(L.load().frg_autotune_table_set(*key_of(p, flux, av, curved), int(variant)), None,
            "frg_autotune_table_set")


def get_variant(p: int, flux: str, av: str, curved: bool = False):
    """The key's variant, or None if the table has no entry for it."""
    v = C.c_int()
    rc = L.load().frg_autotune_table_get(*key_of(p, flux, av, curved), C.byref(v))
    if rc == L.FRG_ERR_STATE:
        return None
    L.check(rc, None, "frg_autotune_table_get")
    return v.value


def clear() -> None:
    L.load().frg_autotune_table_clear()


def size() -> int:
    return int(L.load().frg_autotune_table_size())


def save(path: str) -> None:
    L.check(L.load().frg_autotune_table_save(os.fsencode(path)), None, f"frg_autotune_table_save({path})")


def load(path: str) -> None:
    L.check(L.load().frg_autotune_table_load(os.fsencode(path)), None, f"frg_autotune_table_load({path})")


def load_default() -> bool:
    """Merge the committed B200 table, if present; returns whether it was read."""
    if os.path.exists(DEFAULT_TABLE):
        load(DEFAULT_TABLE)
        return True
    return False


def measure(path: str = DEFAULT_TABLE, ps=(1, 2, 3, 4, 5), fluxes=("hllc", "rusanov"),
            avs=("br0", "local_dd", "none"), reps: int = 3, ctx=None) -> dict:
    """Build the table on this GPU and save it: for every (P, flux,
    dissipation form) of an affine mesh, the autotuner times the tile
    variants on a periodic density wave on a mesh that fills the device
    (512^2 elements for P <= 3, 384^2 above) and records the fastest.
    Returns {"p<P>_<flux>_<av>": variant}."""
    from . import Euler2D, GpuSolve, NullCapturing, PerssonAVMethod
    from .workloads import Workload2D

    out = {}
    for p in ps:
        for flux in fluxes:
            for av in avs:
                n = 512 if p <= 3 else 384
                w = Workload2D("c2", n, p, flux, "null" if av == "none" else "persson_av", 0.1, True, 0.1, 4)
                st, _ = w.build(__import__(__package__))
                m = (NullCapturing() if av == "none" else
                     PerssonAVMethod(c_av=0.1, av_form="element_local_DD" if av == "local_dd" else "conservative_br0"))
                s = GpuSolve(st, Euler2D(1.4), m, ctx=ctx)
                s.upload(st.u, 0.0)
                best, _ = s.autotune(reps=reps)
                out[f"p{p}_{flux}_{av}"] = int(best)
                s.close()
    save(path)
    return out


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="measure the tile table on this GPU and save it as JSON")
    ap.add_argument("--out", default=DEFAULT_TABLE)
    a = ap.parse_args()
    print(json.dumps(measure(a.out)))
