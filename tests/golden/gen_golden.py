"""Generate the golden fixtures from the reference's own FFTW classes.

Runs ONLY in a container that has the reference checkout (default
/root/reference, override with FASTWIGNER_REFERENCE): it loads the
unmodified reference classes through ``oracle/ref_shim.py`` and records
their outputs for the cases of ``tests/golden/cases.py`` into
``tests/golden/*.npz``.  The fixtures are committed; tests never need the
reference tree.

    python tests/golden/gen_golden.py [case ...]
"""
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

from oracle.ref_shim import load_reference  # noqa: E402
from cases import CASES, CONFIG1  # noqa: E402


def run_case(R, case):
    cls = R[case["cls"]]
    kw = dict(case["kw"])
    obj = cls(**kw)
    if case["cls"] == "WignerBlochFFTW1D":
        W = obj.get_gibbs_state()
        return dict(W=np.array(W), num_beta_steps=obj.num_beta_steps, dbeta=obj.dbeta)
    obj.set_wignerfunction(case["init"])
    obj.propagate(case["steps"])
    out = dict(W=np.array(obj.wignerfunction), t=obj.t)
    if obj.isEhrenfest:
        for k in ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average"):
            out[k] = np.array(getattr(obj, k))
    return out


def main():
    R = load_reference(Path(os.environ.get("FASTWIGNER_REFERENCE", "/root/reference")))
    names = sys.argv[1:] or list(CASES) + ["config1_moyal_256"]
    for name in [n for n in names if n in CASES]:
        case = CASES[name]
        out = run_case(R, case)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, {k: np.shape(v) for k, v in out.items()})
    if "config1_moyal_256" not in names:
        return
    out = run_case(R, CONFIG1)
    W = out.pop("W")
    out["W_sum_sq"] = np.sum(W ** 2)
    out["W_row_sums"] = W.sum(axis=1)
    out["W_col_sums"] = W.sum(axis=0)
    np.savez_compressed(HERE / "config1_moyal_256.npz", **out)
    print("config1_moyal_256", {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
