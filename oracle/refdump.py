"""Reader for the text dumps written by ``oracle/_ref/pm_forcedump``.

TEST INFRASTRUCTURE: the dumps are outputs of the unmodified ProtoMol
reference (topology as ProtoMol built it, plus the FP64 forces/energies of
each evaluated force) and pin both the oracle restatement and the CUDA path.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np

from . import System

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
FORCEDUMP = os.path.join(REF_DIR, "pm_forcedump")
PROTOMOL = os.path.join(REF_DIR, "protomol")

# ScalarStructure::Index (type/ScalarStructure.h:26-67)
E_COULOMB, E_LJ, E_BOND, E_ANGLE = 0, 1, 2, 3
E_VIRIAL = 7


def parse(path: str) -> dict:
    out: dict = {"forces": []}
    cur = None
    with open(path) as fh:
        for line in fh:
            toks = line.split()
            if not toks:
                continue
            key, cnt, vals = toks[0], toks[1], toks[2:]
            if key == "typenames":
                out[key] = vals
                continue
            if key == "forcedef":
                cur["def"] = " ".join(vals)
                continue
            if key == "forceid":
                cur["id"] = " ".join(vals)
                continue
            if key == "force":
                cur = {"index": int(vals[0])}
                out["forces"].append(cur)
                continue
            if key in ("type", "molecule", "water", "exclusions", "exclusions_check", "bonds",
                       "angles", "dihedrals", "impropers", "scp_hbond", "scp_residue",
                       "scp_name"):
                arr = np.array([int(v) for v in vals], dtype=np.int64)
            else:
                arr = np.array([float(v) for v in vals], dtype=np.float64)
            if cur is not None and key in ("forces", "energies"):
                cur[key] = arr
            else:
                out[key] = arr
    n = int(out["natoms"][0])
    for f in out["forces"]:
        f["forces"] = f["forces"].reshape(n, 3)
    return out


def to_system(d: dict) -> System:
    n = int(d["natoms"][0])
    nt = int(d["ntypes"][0])
    ex = d["exclusions"].reshape(-1, 3).astype(np.int32)
    table_class = ex[:, 2].copy()
    if "exclusions_check" in d and len(ex):
        ex[:, 2] = d["exclusions_check"].astype(np.int32)
    s = System(
        pos=d["positions"].reshape(n, 3).copy(),
        charge=d["charge"].copy(),
        type=d["type"].astype(np.int32),
        molecule=d["molecule"].astype(np.int32),
        lj=d["lj"].reshape(nt, nt, 4).copy(),
        excl=ex,
        coulomb_scaling=float(d["coulomb_scaling"][0]),
        periodic=bool(int(d["periodic"][0])),
        box=d["box"].copy(),
        mass=d["mass"].copy(),
        water=d["water"].astype(np.int32),
        excl_table_class=table_class,
    )
    if "scp_alpha" in d:
        s.scpism = {k: d[k].copy() for k in d if k.startswith("scp_")}
    if "gb_vdwr" in d:
        s.gb_vdwr = d["gb_vdwr"].copy()
        s.gb_scale = d["gb_scale"].copy()
        s.gb_offset = d["gb_offset"].copy()
        s.gb_obc = tuple(d["gb_obc"])
    return s


def run(conf: str, out: str, forces: list[str], steps: int = 0, cwd: str | None = None):
    """Run the reference's force dump on a conf (test-time only)."""
    cmd = [FORCEDUMP, conf, out]
    if steps:
        cmd += ["--steps", str(steps)]
    cmd += forces
    subprocess.run(cmd, cwd=cwd, check=True, stdout=subprocess.DEVNULL,
                   stderr=subprocess.DEVNULL)
    return parse(out)
