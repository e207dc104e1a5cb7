"""Generate the golden fixtures that pin the oracle to the reference.

Run where the reference tree is checked out, with its root in REF, after
oracle/_ref has been built from it:

    make -C oracle REF=<reference root>
    REF=<reference root> python tests/golden/make_golden.py

Writes tests/golden/reference_pins.npz and reference_pins.json:
  * sort_*      : the reference's own local key sort (sl_pepc sort_radix.c,
                  compiled from its sources into oracle/_ref) run on seeded key
                  sets, including heavy duplicates -> sorted keys and the
                  0-based permutation (tie order included)
  * lattice_*   : the pretabulated unit-cube lattice coefficients of
                  load_lattice_coefficients (coulomb/module_fmm_framework.f90:260-508),
                  parsed from the source text
  * par_rand_kat: the documented first draws of pepc-mini's generator
                  (frontends/pepc-mini/module_helper.f90:586-590)
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

REF = os.environ.get("REF")


def sort_sets():
    rng = np.random.default_rng(20261203)
    sets = {}
    # distinct level-20 keys: placeholder bit 60 set
    sets["distinct"] = rng.integers(1 << 60, 1 << 61, size=6000, dtype=np.int64)
    # heavy duplicates (ties exercise the unstable in-place MSD order)
    base = rng.integers(1 << 60, 1 << 61, size=700, dtype=np.int64)
    sets["dups"] = base[rng.integers(0, 700, size=6000)]
    # the first 10-bit digit (bits 54..63) has 64 live classes for level-20
    # keys, so 40000 keys put > 256 keys in a class and exercise the recursion
    sets["large"] = rng.integers(1 << 60, 1 << 61, size=40000, dtype=np.int64)
    return sets


def lattice_table():
    path = os.path.join(REF, "src/interaction_specific/coulomb/module_fmm_framework.f90")
    txt = open(path).read()
    body = txt[txt.index("subroutine load_lattice_coefficients"):]
    body = body[:body.index("end subroutine load_lattice_coefficients")]
    pat = re.compile(r"M\(tblinv\(\s*(\d+),\s*(\d+),\s*Lmax_taylor\)\)\s*=\s*([-+0-9.E]+)_kind_physics")
    ls, ms, vs = [], [], []
    for m in pat.finditer(body):
        ls.append(int(m.group(1)))
        ms.append(int(m.group(2)))
        vs.append(float(m.group(3)))
    return np.array(ls), np.array(ms), np.array(vs)


def par_rand_kat():
    path = os.path.join(REF, "src/frontends/pepc-mini/module_helper.f90")
    txt = open(path).read()
    m = re.search(r"first numbers should be ([0-9.]+), ([0-9.]+) and ([0-9.]+)", txt)
    return np.array([float(m.group(i)) for i in (1, 2, 3)])


def main():
    if not REF or not os.path.isdir(REF):
        raise SystemExit("set REF to the root of the reference checkout")
    out = {}
    prov = {"reference": "ALaDyn/pepc", "sort": "oracle/_ref/libslref.so (sl_pepc sort_radix.c)"}
    for name, keys in sort_sets().items():
        r = O.ref_sort(keys)
        if r is None:
            raise SystemExit("oracle/_ref/libslref.so not built: run make -C oracle")
        assert np.array_equal(keys[r[1]], r[0])
        out[f"sort_{name}_in"] = keys
        out[f"sort_{name}_idx"] = r[1].astype(np.int32)
    ls, ms, vs = lattice_table()
    out["lattice_l"], out["lattice_m"], out["lattice_v"] = ls, ms, vs
    out["par_rand_kat"] = par_rand_kat()
    np.savez_compressed(os.path.join(HERE, "reference_pins.npz"), **out)
    prov["lattice_entries"] = int(len(vs))
    prov["par_rand_kat"] = out["par_rand_kat"].tolist()
    with open(os.path.join(HERE, "reference_pins.json"), "w") as fh:
        json.dump(prov, fh, indent=1)
    print("wrote", os.path.join(HERE, "reference_pins.npz"), {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
