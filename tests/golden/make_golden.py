"""Extract the reference's golden end-to-end vectors into tests/golden/.

Source: bfps/test/B32p1e4_checkpoint_0.h5, the fixture of the reference's
only asserting regression test (bfps/test/test_bfps_NSVEparticles.py:12-52):
NSVEparticles, N=32, single precision, 10^4 tracers with beta_n1_m1, AB4,
run as two jobs of 32 steps.  libhdf5/h5py are not available; the file is
read through its groups by bfps_b200.h5, and the contents are checked (the
IC positions equal ``np.random.seed(2); np.random.random((10000,3))*2*pi``
bit for bit, the shifted rhs[0] is zero, the fields are Hermitian on the
kx=0 plane at iterations 32 and 64, which were written after symmetrize).

Run from the repository root:  python tests/golden/make_golden.py
Writes tests/golden/B32p1e4.npz.
"""
import os
import sys
import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from bfps_b200 import h5  # noqa: E402

SRC = os.path.join(os.environ.get("BFPS_REFERENCE", "/root/reference"), "bfps", "test",
                   "B32p1e4_checkpoint_0.h5")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "B32p1e4.npz")

DATASETS = ["vorticity/complex/0", "vorticity/complex/32", "vorticity/complex/64",
            "tracers0/state/0", "tracers0/state/32", "tracers0/state/64",
            "tracers0/rhs/32", "tracers0/rhs/64"]

# number of tracers kept in the committed fixture (tracers are independent
# given the field, so a prefix is an exact sub-check of the full comparison)
NKEEP = 2000


def read_all(path=SRC):
    with h5.File(path, "r") as f:
        return {name: f[name][()] for name in DATASETS}


def validate(d):
    np.random.seed(2)
    ic = np.random.random((10000, 3)) * 2 * np.pi
    assert np.array_equal(d["tracers0/state/0"], ic), "state/0 offset"
    for it in (32, 64):
        r = d["tracers0/rhs/%d" % it]
        assert np.all(r[0] == 0) and np.all(np.isfinite(r)), "rhs/%d offset" % it
        assert np.abs(r[1]).max() > 0.1
        s = d["tracers0/state/%d" % it]
        assert np.all(np.isfinite(s)) and np.abs(s - ic).max() < 2.0
    assert np.all(np.isfinite(d["vorticity/complex/0"]))
    for it in (32, 64):
        # written after field::symmetrize, so exactly Hermitian on kx = 0
        v = d["vorticity/complex/%d" % it]
        assert np.all(np.isfinite(v))
        plane = v[:, :, 0, :]
        herm = np.conj(plane[(-np.arange(32)) % 32][:, (-np.arange(32)) % 32])
        assert np.abs(plane - herm)[1:16].max() == 0, "field %d" % it


def main():
    d = read_all()
    validate(d)
    keep = {}
    for it in (0, 32, 64):
        keep["vorticity_%d" % it] = d["vorticity/complex/%d" % it]
    for it in (32, 64):
        keep["state_%d" % it] = d["tracers0/state/%d" % it][:NKEEP]
        keep["rhs_%d" % it] = d["tracers0/rhs/%d" % it][:, :NKEEP]
    np.savez_compressed(OUT, **keep)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    sys.exit(main())
