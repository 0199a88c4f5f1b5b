"""Data formats (CPU): the reference's .mat amplitude table through
load_amplitude_table, and the on-disk path-record format round trip."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mcspeckle_b200 import formats as F
from mcspeckle_b200 import mc as MC


def test_amplitude_table_from_mat_matches_reference_fixture(tmp_path):
    """A .mat written with the fixture's theta / farField loads into the
    tables the reference built from scatteringAmplitude.mat."""
    import scipy.io as sio
    z = np.load(os.path.join(GOLDEN, "table_2d_scatteringAmplitude.npz"))
    p = tmp_path / "amp.mat"
    sio.savemat(p, {"theta": z["theta"].reshape(1, -1), "farField": z["f"].reshape(1, -1)})
    st = F.load_amplitude_table(str(p))
    for k in ("evalAmp", "sampleIcdf"):
        a = np.asarray(st["ampfunc"][k]).reshape(-1)
        b = np.asarray(z["out_" + k]).reshape(-1)
        assert np.max(np.abs(a - b)) <= 1e-9 * max(1.0, np.max(np.abs(b)))


def test_amplitude_table_missing_variables(tmp_path):
    import scipy.io as sio
    p = tmp_path / "bad.mat"
    sio.savemat(p, {"angles": np.zeros((1, 3))})
    with pytest.raises(KeyError):
        F.load_amplitude_table(str(p))


def test_record_file_round_trip(tmp_path, oracle_lib):
    """Records from the oracle's walk, written and read back, keep every
    field, carry the arguments to rebuild the solve, and replay (oracle FP64
    accumulation) to the oracle's own field."""
    O = oracle_lib
    from cases import small_cases
    name, args, extra = small_cases(80)[4]  # tabulated, ampfunc0
    h = MC.mc_args(*(args + extra), seed=21, precision="fp64")
    o = O.records(h, O.Rng.philox(), True, 100000)
    r = MC.Records(o.n)
    for k in ("x", "ow", "x1", "w1", "wpx", "xi", "plen", "path"):
        setattr(r, k, np.ascontiguousarray(getattr(o, k)))
    r.n = o.n
    p = tmp_path / "rec.npz"
    F.save_records(str(p), r, h)
    r2, meta, arrays = F.load_records(str(p))
    for k in ("x", "ow", "x1", "w1", "wpx", "xi", "plen", "path"):
        assert np.array_equal(getattr(r2, k), getattr(r, k))
    h2 = F.args_from_records(meta, arrays)
    assert h2.args.nl == h.args.nl and h2.args.nv == h.args.nv and h2.args.has_ampfunc0
    u_rep = O.field_from_records(h2, r2)
    u = O.field(h, O.Rng.philox())
    assert np.max(np.abs(u_rep - u)) <= 1e-10 * np.max(np.abs(u))


def test_record_file_rejects_other_files(tmp_path):
    p = tmp_path / "x.npz"
    np.savez(p, meta='{"format": "other"}')
    with pytest.raises(ValueError):
        F.load_records(str(p))
