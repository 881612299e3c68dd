"""Golden vectors of the reference's initial vector field, for the launcher.

bfps.DNS.generate_vector_field (bfps/DNS.py:734-806) seeds numpy's legacy
generator with 7547, draws three components with bfps.tools.generate_data_3D
(bfps/tools.py:96-144) on the half grid and embeds them with
bfps.tools.padd_with_zeros (bfps/tools.py:169-203); DNS.launch_jobs calls it
with spectra_slope=2 and amplitude=0.05 when no source field is given
(bfps/DNS.py:866-869).  This script runs the reference's own tools module
(loaded from the reference checkout; its module-level `import h5py` and a
default argument naming an h5py type, unused by these two functions, are
satisfied by a stand-in) and stores the 16^3 single-precision field.

Run from the repository root:  python tests/golden/make_ic_golden.py
Writes tests/golden/ic_vector_field_n16.npz.
"""
import importlib.util
import os
import sys
import types

import numpy as np

TOOLS = os.path.join(os.environ.get("BFPS_REFERENCE", "/root/reference"), "bfps", "tools.py")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ic_vector_field_n16.npz")
N = 16


def main():
    stand_in = types.ModuleType("h5py")
    stand_in.h5t = types.SimpleNamespace(IEEE_F64LE=None)
    sys.modules.setdefault("h5py", stand_in)
    spec = importlib.util.spec_from_file_location("reference_tools", TOOLS)
    tools = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(tools)
    np.random.seed(7547)
    comps = [tools.generate_data_3D(N // 2, N // 2, N // 2, p=2.0, amplitude=0.05).astype(np.complex64)
             for _ in range(3)]
    k0 = np.zeros(comps[0].shape + (3,), comps[0].dtype)
    for i in range(3):
        k0[..., i] = comps[i]
    field = tools.padd_with_zeros(k0, N, N, N)
    np.savez_compressed(OUT, field=field)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    sys.exit(main())
