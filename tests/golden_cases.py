"""Loader for the golden fixtures in tests/golden (made by make_golden.py)."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILTER_CODES = {"shlo": 1, "shepp": 1, "hann": 2, "hamm": 3, "hamming": 3, "ramp": 4,
                "ramlak": 4, "none": 0}


def cases():
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "case_*.npz"))):
        z = dict(np.load(f))
        case = {"name": os.path.basename(f)[5:-4], "sino1": z["sino1"], "sino2": z["sino2"],
                "theta": z["theta"], "n_det": int(z["n_det"]), "n_ang": int(z["n_ang"]),
                "center": float(z["center"]), "sampl": float(z["sampl"]), "C": float(z["C"]),
                "M0": int(z["M0"]), "geom": int(z["geom"]) if "geom" in z else 0,
                "roi": tuple(float(v) for v in z["roi"]) if "roi" in z else (1.0, 1.0, 0.0, 0.0)}
        if str(z["kind"]) == "gridrec":
            case["filter"] = int(z["filter"])
            case["ref32"] = (z["ref32_1"], z["ref32_2"])
            case["ref64"] = (z["ref64_1"], z["ref64_2"])
        else:
            case["filter"] = FILTER_CODES[str(z["filter_name"])]
            case["ref32"] = (z["refb_1"], z["refb_2"])
            case["ref64"] = None
        out.append(case)
    return out
