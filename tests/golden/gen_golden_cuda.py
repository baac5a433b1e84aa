"""Generate golden fixtures from the reference's own CUDA classes.

Runs ONLY in a container that has the reference checkout (default
/root/reference, override with FASTWIGNER_REFERENCE) and g++: it loads the
unmodified reference classes RhoVNeumannCUDA1D, RhoBlochCUDA1D,
WignerMoyalCUDA1D and WignerBlochCUDA1D through ``oracle/ref_cuda_shim.py``
(their kernel strings compiled for the host CPU, cuFFT replaced by pocketfft
with cuFFT's unnormalised conventions) and records their outputs for the cases
of ``tests/golden/cases_cuda.py`` into ``tests/golden/cuda_*.npz``.  The
fixtures are committed; tests never need the reference tree.

    python tests/golden/gen_golden_cuda.py [case ...]
"""
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

from cases_cuda import CUDA_CASES  # noqa: E402
from oracle.ref_cuda_shim import load_reference_cuda  # noqa: E402

OBS = ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average")


def run_case(R, case):
    import pycuda.gpuarray as gpuarray  # the host stand-in installed by load_reference_cuda

    obj = R[case["cls"]](**dict(case["kw"]))
    out = {}
    if case["cls"].startswith("Rho"):
        if "gibbs" in case:
            obj.get_gibbs_state(**case["gibbs"])
        elif "ground" in case:
            obj.get_ground_state(**case["ground"])
        else:
            obj.set_rho(case["init"])
            out["rho0"] = obj.rho.get()
            if case.get("wigner_time"):
                obj.wigner_initial = gpuarray.to_gpu(np.ascontiguousarray(obj.get_wignerfunction().get().real))
                out["wigner_initial"] = obj.wigner_initial.get()
            obj.propagate(case["steps"])
            out["t"] = float(obj.t)
            for k in OBS + ("wigner_time",):
                if hasattr(obj, k):
                    out[k] = np.array(getattr(obj, k))
        out["rho"] = obj.rho.get()
        out["purity"] = float(obj.get_purity())
        out["W"] = obj.get_wignerfunction().get()
        out["sigma_x_sigma_p"] = float(obj.get_sigma_x_sigma_p())
        return out
    if case["cls"] == "WignerBlochCUDA1D":
        if "gibbs" in case:
            out["W_gibbs"] = obj.get_gibbs_state(**case["gibbs"]).get()
        if "ground" in case:
            out["W_ground"] = obj.get_ground_state(**case["ground"]).get()
            out["purity_ground"] = float(obj.get_purity())
        return out
    obj.set_wignerfunction(case["init"])
    out["W0"] = obj.wignerfunction.get()
    obj.propagate(case["steps"])
    out["t"] = float(obj.t)
    out["W"] = obj.wignerfunction.get()
    for k in OBS:
        if hasattr(obj, k):
            out[k] = np.array(getattr(obj, k))
    out["purity"] = float(obj.get_purity())
    return out


def main():
    R = load_reference_cuda(Path(os.environ.get("FASTWIGNER_REFERENCE", "/root/reference")))
    names = sys.argv[1:] or list(CUDA_CASES)
    for name in names:
        out = run_case(R, CUDA_CASES[name])
        np.savez_compressed(HERE / f"cuda_{name}.npz", **out)
        print(name, {k: np.shape(v) for k, v in out.items()}, flush=True)


if __name__ == "__main__":
    main()
