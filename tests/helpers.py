"""Shared helpers for the parity tests: golden fixtures and System construction."""
import ast
import os

import numpy as np

from coupled_cluster_doubles_b200 import System

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SMALL = ["pairing_gm1.0", "pairing_gm0.5", "pairing_gp0.5", "pairing_gp1.0", "pnm14_s4",
         "snm4_s4", "eg14_s19"]
# Further reference runs that pin the builder and the oracle (CPU tests).
EXTRA = ["eg14_r05", "eg14_r2", "pnm14_d016", "pairing_l6n4", "eg38_s16"]
STRUCT = ["chan_dims", "chan_mod_dims", "three_body_dims", "pp_map", "hh_map", "ph_mod_map",
          "hp_mod_map", "hpp_map", "phh_map", "sp_energy"]
MAPS = ["map_iab_j", "map_jab_i", "map_a_bij", "map_b_aij", "map_ai_jb", "map_aj_ib",
        "map_bi_ja", "map_bj_ia"]
VKINDS = ["v_hhhh", "v_hhpp", "v_pppp", "v_hpph_mod", "v_hphp_mod", "v_h_hpp", "v_phh_p"]


def golden(name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    g["params"] = ast.literal_eval(str(g["params"]))
    g["kind"] = str(g["kind"])
    g["tol"] = float(g["scalars"][3])
    return g


def system_for(g, load_v_pppp=True):
    return getattr(System, g["kind"])(**g["params"], load_v_pppp=load_v_pppp)


def t2_sample(g, t2):
    return t2 if int(g["t2_full"][0]) else t2[::97]
