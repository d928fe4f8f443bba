"""Element parameter table reader (format of SPAMMM data/ElementTypes.dat).

Mirrors ``read_element_types`` (spammm/topology/FFparams.py:103-143): one
whitespace-separated row per element, ``#`` comments; columns
name iZ ne nv npi color Rcov RvdW EvdW Quff Uuff Vuff [Eaff Ehard Ra eta].
"""
import os
from dataclasses import dataclass

DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "ElementTypes.dat")


@dataclass
class ElementType:
    name: str
    iZ: int = 0
    neval: int = 0
    valence: int = 0
    piMax: int = 0
    color: int = 0
    Rcov: float = 0.0
    RvdW: float = 0.0
    EvdW: float = 0.0
    Quff: float = 0.0
    Uuff: float = 0.0
    Vuff: float = 0.0


def read_element_types(filepath=None):
    """dict element-name -> ElementType."""
    out = {}
    with open(filepath or DEFAULT_PATH, "r") as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            p = line.split()
            et = ElementType(name=p[0])
            et.iZ = int(p[1])
            et.neval = int(p[2])
            et.valence = int(p[3])
            et.piMax = int(p[4])
            et.color = int(p[5], 16) if p[5].startswith("0x") else int(p[5])
            et.Rcov = float(p[6])
            et.RvdW = float(p[7])
            et.EvdW = float(p[8])
            et.Quff = float(p[9])
            et.Uuff = float(p[10])
            et.Vuff = float(p[11])
            out[et.name] = et
    return out


def z_map(types):
    """dict atomic number -> ElementType."""
    return {int(e.iZ): e for e in types.values()}
