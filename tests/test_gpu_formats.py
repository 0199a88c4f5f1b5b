"""Path records on disk, replayed on the GPU (scmc_field_from_records):
records exported from the GPU walk, written in the record format and read
back, give the GPU field of the same solve (FP64 1e-10, mixed 1e-3)."""
import numpy as np
import pytest

from cases import small_cases
from mcspeckle_b200 import formats as F
from mcspeckle_b200 import mc as MC

pytestmark = pytest.mark.gpu

CASES = small_cases(250)


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.parametrize("idx", [0, 2, 3, 4, 6])
def test_records_file_replays_to_the_field(gpu, tmp_path, idx):
    name, args, extra = CASES[idx]
    h = MC.mc_args(*(args + extra), seed=31, precision="fp64")
    r = MC.export_records(h, True, 50000)
    p = tmp_path / f"{name}.npz"
    F.save_records(str(p), r, h)
    u = MC.field_from_args(h)
    assert rel(F.replay_field(str(p)), u) < 1e-10
    assert rel(F.replay_field(str(p), precision="mixed"), u) < 1e-3
