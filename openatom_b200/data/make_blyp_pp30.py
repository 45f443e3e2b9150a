"""Write blyp_pp30.npz: the radial tables of the reference's shipped O and H
pseudopotentials (data/DATABASE/O_BLYP_PP30.pseud, H_BLYP_PP30.pseud; the
O/H entries of data/DATABASE/pi_md.vps: O KB with N_ANG 1, LOC_OPT 1; H LOC
with N_ANG 0, LOC_OPT 0), read with openatom_b200.pseudo.read_pseud, so that
systems can be built where the reference tree is absent.

Run from the repository root:  python openatom_b200/data/make_blyp_pp30.py [reference root]
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from openatom_b200.pseudo import read_pseud  # noqa: E402

ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
out = {}
for name in ("O", "H"):
    pp = read_pseud(os.path.join(ref, "data", "DATABASE", f"{name}_BLYP_PP30.pseud"))
    for k in ("nr", "rmax", "nang", "z1", "a1", "z2", "a2", "zpol", "gamma"):
        out[f"{name}_{k}"] = np.array(pp[k])
    out[f"{name}_v"] = pp["v"]
    out[f"{name}_rphi"] = pp["rphi"]
np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "blyp_pp30.npz"), **out)
