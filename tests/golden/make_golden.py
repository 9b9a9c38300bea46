"""Writes tests/golden/reference_kats.json: the known-answer vectors of the
reference's own tests, transcribed as data (inputs and expected outputs), so
that the oracle and the engine are pinned to them without reading the
reference tree at test time.

Sources (AFQMCLAB project root):
  afqmc/blocks/walker/SD/test/SDTest.cpp:158-173
  afqmc/blocks/walker/SD2s/test/SD2sTest.cpp:183-200
  afqmc/blocks/walker/SD2is/test/SD2isTest.cpp:164-178
  afqmc/blocks/oneBodyWalkerOperation/logHop2isSD2isOperation/test/logHop2isSD2isOperationTest.cpp:25-94
  afqmc/utilities/populationControl/test/populationControlTest.cpp:12-45

Run from the repository root: python tests/golden/make_golden.py
(the values below are typed in from those files; the script only reshapes them).
"""
import json
import os

# column-major complex entries as (re, im) pairs
WF_4x3 = [(1, 1), (2, 1), (3, 1), (4, 1), (2, 2), (3, 1), (5, 2), (6, 1), (4, 1), (3, 3), (2, 2),
          (2, 6)]
WF_DN_4x2 = [(1, 2), (2, 3), (3, 4), (4, 5), (2, 2), (3, 3), (5, 2), (6, 3)]
TAYLOR_M = [(2, 3), (4, 2), (1, 1), (1, -1), (0, 0.3), (1, -1), (3, 2), (2, 3), (0, 0.5)]
TAYLOR_WF = [(1, 0), (2, 0), (3, 0), (3, 0), (4, 0), (5, 0)]
TAYLOR_RIGHT = [(0.8717255743431891, -0.06695756061260984), (1.9019539751922434, -0.11272541520548454),
                (2.9713563453236675, -0.0038676809054978764), (2.753351116138562, -0.14393925193667553),
                (3.7836486105153155, -0.21511811236274694), (4.932649990968739, -0.012861814634312912)]
TAYLOR_LEFT = [(0.8708226627963166, 0.09656591603485742), (1.961995737773784, -0.034019035572233965),
               (2.9316294741182647, 0.09182786294989435), (2.7315235332357157, 0.21256279549696155),
               (3.924363675467334, -0.0680085413131974), (4.833174488748831, 0.19818901143889675)]
# one-based parent table for weights 1..100 over 4 ranks
POP_TABLE = [60, 62, 66, 69, 71, 73, 75, 8, 77, 80, 82, 82, 13, 14, 84, 85, 87, 88, 90, 20, 92, 22,
             23, 92, 25, 32, 44, 28, 93, 30, 94, 32, 96, 34, 35, 97, 37, 38, 39, 40, 98, 42, 99, 44,
             45, 100, 47, 48, 49, 50, 51, 52, 53, 53, 55, 56, 57, 58, 59, 60, 55, 62, 63, 64, 65,
             66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 77, 78, 79, 80, 81, 82, 83, 84, 85, 86,
             87, 88, 89, 90, 91, 92, 93, 94, 95, 96, 97, 98, 99, 100]

data = {
    "sd_normalize": {"shape": [4, 3], "wf": WF_4x3, "logw": 3.35769169316734,
                     "ratio": 0.19286583895005868},
    "sd2is_normalize": {"shape": [4, 3], "nup": 3, "ndn": 2, "wf": WF_4x3,
                        "logw": 5.2382917510141205, "ratio": 0.19286583895005868},
    "sd2s_normalize": {"shape_up": [4, 3], "shape_dn": [4, 2], "wf_up": WF_4x3,
                       "wf_dn": WF_DN_4x2, "logw": 5.83560522196797,
                       "ratio": 0.14186161056920224},
    "loghop_taylor": {"M_scale": -0.01, "M": TAYLOR_M, "wf": TAYLOR_WF, "right": TAYLOR_RIGHT,
                      "left": TAYLOR_LEFT, "fixed_order": 8, "fixed_tol": 1e-12,
                      "auto_accuracy": 1e-8, "auto_order": 6, "auto_tol": 1e-8},
    "pop_configuration": {"L": 100, "size": 4, "weights": "i+1", "table_one_based": POP_TABLE,
                          "note": "SPRNG seed 985456376; only the slot-filling half is pinnable"},
    "pop_check": [{"weights": [float(i + 1) for i in range(10)], "min": 1.0, "max": 10.0,
                   "avg": 5.5},
                  {"weights": [1.0] * 5 + [6.0] + [1.0] * 4, "min": 1.0, "max": 6.0,
                   "avg": 1.5}],
}

if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(out, "w") as f:
        json.dump(data, f, indent=1)
    print(out)
