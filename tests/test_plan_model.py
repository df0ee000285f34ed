"""The plan-variant network compiled into the library (csrc/plan_model.cpp)
is the committed model (selector_data/plan_model.npz), weight for weight, and
was trained for the library's variant list."""
import json
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def test_compiled_weights_are_the_committed_model():
    z = np.load(ROOT / "sparsep_b200" / "selector_data" / "plan_model.npz")
    src = (ROOT / "sparsep_b200" / "csrc" / "plan_model.cpp").read_text()
    body = src[src.index("kWb["):src.index("};")]
    wb = np.array([int(v, 16) for v in re.findall(r"0x([0-9a-f]{4})", body)], dtype=np.uint16)
    assert np.array_equal(wb, z["wb"].astype(np.uint16))
    for name, key in (("kMean", "mean"), ("kStd", "std")):
        line = next(ln for ln in src.splitlines() if ln.startswith(f"const float {name}"))
        vals = np.array([float(v.rstrip("f")) for v in re.findall(r"[-+0-9.e]+f", line.split("=", 1)[1])],
                        dtype=np.float32)
        assert np.array_equal(vals, z[key].astype(np.float32)), name


def test_model_metadata():
    z = np.load(ROOT / "sparsep_b200" / "selector_data" / "plan_model.npz")
    meta = json.loads(str(z["meta"]))
    assert len(meta["variants"]) == 10 and meta["variants"][0] == "csr/1d/auto"
    assert meta["heldout_eval"]["regret_total"] <= 0.10
