"""The tuning table (scmc_tuning_*): entries from a file or set directly,
resolved per (kind, precision, size) with the built-in defaults filled in;
the last matching entry wins; bad files are refused.  No GPU needed."""
import ctypes as C

import pytest

from mcspeckle_b200 import _abi, _lib


@pytest.fixture()
def L():
    L = _lib.lib()
    _lib.check(L.scmc_tuning_clear())
    yield L
    _lib.check(L.scmc_tuning_clear())


def get(L, kind, prec, n):
    t = _abi.Tuning()
    _lib.check(L.scmc_tuning_get(kind, prec, n, C.byref(t)))
    return t


def test_defaults_and_file_entries(L, tmp_path):
    t = get(L, _abi.SCMC_TUNE_COV, _abi.PRECISIONS["fp16"], 4096)
    assert (t.path_batch, t.chunk_events, t.stages, t.ksplit, t.group_entries) == (1 << 20, 0, 2, 0, 1 << 20)
    f = tmp_path / "tune.txt"
    f.write_text("# kind precision n_lo n_hi path_batch chunk_events stages ksplit group_entries\n"
                 "cov fp16 1000 5000 524288 32768 3 0 0\n"
                 "cov fp16 4096 4096 0 0 2 0 0   # a later, narrower entry wins for its fields\n"
                 "field mixed 1 100000 0 0 0 4 0\n"
                 "fq fp16 65536 65536 0 0 0 0 262144\n")
    _lib.check(L.scmc_tuning_load(str(f).encode()))
    t = get(L, _abi.SCMC_TUNE_COV, _abi.PRECISIONS["fp16"], 4096)
    assert (t.path_batch, t.chunk_events, t.stages) == (524288, 32768, 2)
    t = get(L, _abi.SCMC_TUNE_COV, _abi.PRECISIONS["fp16"], 2000)
    assert t.stages == 3
    assert get(L, _abi.SCMC_TUNE_COV, _abi.PRECISIONS["mixed"], 4096).chunk_events == 0
    assert get(L, _abi.SCMC_TUNE_FIELD, _abi.PRECISIONS["mixed"], 256).ksplit == 4
    assert get(L, _abi.SCMC_TUNE_FQ, _abi.PRECISIONS["fp16"], 65536).group_entries == 262144


def test_set_and_bad_input(L, tmp_path):
    t = _abi.Tuning(kind=_abi.SCMC_TUNE_FIELD, precision=_abi.PRECISIONS["fp16"], n_lo=1, n_hi=10, path_batch=4096)
    _lib.check(L.scmc_tuning_set(C.byref(t)))
    assert get(L, _abi.SCMC_TUNE_FIELD, _abi.PRECISIONS["fp16"], 5).path_batch == 4096
    assert get(L, _abi.SCMC_TUNE_FIELD, _abi.PRECISIONS["fp16"], 11).path_batch == 1 << 20
    bad = _abi.Tuning(kind=7)
    assert L.scmc_tuning_set(C.byref(bad)) == _abi.SCMC_ERR_INVALID
    f = tmp_path / "bad.txt"
    f.write_text("cov fp16 1 2 3\n")
    assert L.scmc_tuning_load(str(f).encode()) == _abi.SCMC_ERR_INVALID
    assert L.scmc_tuning_load(str(tmp_path / "missing.txt").encode()) == _abi.SCMC_ERR_INVALID
