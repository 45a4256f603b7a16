"""The bed generator CLI writes reference input directories that the
library's own solv.txt reader accepts (no GPU needed)."""
import ctypes as C
import json
import os

import pytest

from fluidized_bed_master_b200.beds import _cli
from fluidized_bed_master_b200.params import SphdemParams


@pytest.mark.parametrize("bed,sets", [("box_bed", ["n_fluid=3000", "n_dem=200"]),
                                      ("isph_column", ["dx=2.0e-2"]),
                                      ("dam_break_2d", ["dx=2.0e-2"])])
def test_cli_writes_a_readable_input_dir(tmp_path, bed, sets):
    out = str(tmp_path / bed)
    assert _cli([bed, "--out", out, "--seed", "5", "--set", *sets]) == 0
    for f in ("input.txt", "solv.txt", "data.txt", "params.json"):
        assert os.path.isfile(os.path.join(out, f)), f
    with open(os.path.join(out, "input.txt")) as fh:
        label = fh.readline().split()
        rows = [ln for ln in fh if ln.strip()]
    assert label[:3] == ["1", "2", "3"] and len(rows) > 0
    assert all(len(r.split()) == len(label) for r in rows[:50])
    want = json.load(open(os.path.join(out, "params.json")))
    from fluidized_bed_master_b200.engine import lib

    L = lib()
    L.sphdem_read_solv.argtypes = [C.c_char_p, C.POINTER(SphdemParams)]
    got = SphdemParams()
    assert L.sphdem_read_solv(os.path.join(out, "solv.txt").encode(), C.byref(got)) == 0
    for k in ("kernel_type", "dim", "solver_type", "kgc_solve", "xsph_solve", "freq_filt"):
        assert getattr(got, k) == want[k], k
    for k in ("kappa", "dt", "soundspeed"):
        assert abs(getattr(got, k) - want[k]) <= 1e-12 * max(1.0, abs(want[k])), k
