"""Host-side checks that need no GPU: the C ABI library loads and exports
every declared entry point, the parameter struct layout and the
reference-compat preset, the solv.txt and input.txt readers, and the
status codes of calls that fail before touching a device."""
import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

from fluidized_bed_master_b200 import beds
from fluidized_bed_master_b200.engine import SphdemError, default_params, lib, read_input_txt, read_solv
from fluidized_bed_master_b200.params import SphdemParams, reference_params
from oracle import REFERENCE_DIR

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "sphdem.h")


def declared():
    src = open(HDR).read()
    return sorted(set(re.findall(r"\b(sphdem_[a-z_0-9]+)\s*\(", src)))


def test_exports_every_declared_symbol():
    L = lib()
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_params_layout_and_preset():
    L = lib()
    assert L.sphdem_params_size() == C.sizeof(SphdemParams)
    d = default_params().as_dict()
    r = reference_params().as_dict()
    assert {k for k in d if d[k] != r[k]} == set()
    # values the reference hard-wires (Parameters.cuh, functions_PROP.cuh, functions_NNPS.cuh:2-5)
    p = default_params()
    assert p.rho_gas == 1.784 and p.mu_gas == 2.0e-5 and p.g_sph == 9.8 and p.h_over_dx == 1.6
    assert (p.obc_L1, p.obc_L2, p.obc_L3, p.obc_L4) == (-10.505, -0.021, 0.006, 10.25)
    assert p.dem_shear_modulus == 8.3e8 and p.dem_poisson == 0.23 and p.cyl_r == 0.0125


def test_solv_roundtrip():
    p = reference_params()
    p.kernel_type = 3
    p.con_solve = 1
    p.dt = 1.25e-6
    p.freq_filt = 17
    p.margin[4] = 0.25
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "solv.txt")
        beds.write_solv_txt(path, p)
        q = read_solv(path)
    for k in ("solver_type", "dim", "kernel_type", "rho_type", "time_type", "open_boundary", "fp_solve",
              "fv_solve", "fg_solve", "con_solve", "xsph_solve", "kgc_solve", "delSPH_solve", "freq_filt",
              "freq_output", "decouple_stride", "kappa", "dt", "u_limit", "c_xsph", "soundspeed", "rho0_eos"):
        assert getattr(q, k) == getattr(p, k), k
    assert q.margin[4] == 0.25


@pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE_DIR, "input", "solv.txt")),
                    reason="reference tree not present")
def test_parses_reference_solv():
    q = read_solv(os.path.join(REFERENCE_DIR, "input", "solv.txt"))
    assert q.solver_type == 1 and q.dim == 3 and q.kernel_type == 5 and q.kgc_solve == 1
    assert q.delSPH_solve == 2 and q.xsph_solve == 1 and q.open_boundary == 1 and q.con_solve == 0
    assert q.dt == 5.0e-7 and q.kappa == 2.0 and q.freq_filt == 40 and q.u_limit == 40.0 and q.c_xsph == 0.1


def test_input_txt_reader_matches_generator():
    p, sph, dem = beds.spouted_bed(dx=3.0e-3, n_dem=50, r_dem=1.0e-3, seed=3)
    with tempfile.TemporaryDirectory() as d:
        beds.write_input_dir(d, p, sph, dem)
        s2, d2 = read_input_txt(os.path.join(d, "input.txt"))
    assert len(s2["x"]) == len(sph["x"]) and len(d2["x"]) == len(dem["x"])
    for f in ("x", "y", "z", "h", "m", "rho", "temp"):
        assert np.array_equal(s2[f], np.asarray(sph[f], dtype=float)), f
    for f in ("x", "rad", "ri", "m"):
        assert np.array_equal(d2[f], dem[f]), f
    assert np.array_equal(s2["p_type"], sph["p_type"]) and np.array_equal(d2["dem_idx"], dem["dem_idx"])


def test_malformed_input_rejected():
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "input.txt")
        with open(path, "w") as fh:
            fh.write("1\t2\t3\t8\n0.1 0.2 0.3 1\n0.1 0.2\n")   # truncated last row
        with pytest.raises(SphdemError) as e:
            read_input_txt(path)
        assert e.value.status == -3
        with open(path, "w") as fh:
            fh.write("1\t2\t99\n0 0 0\n")                        # unknown column label
        with pytest.raises(SphdemError):
            read_input_txt(path)


def test_failures_before_the_device():
    L = lib()
    p = default_params()
    h = C.c_void_p()
    assert L.sphdem_create(None, 10, 0, C.byref(h)) == -1
    assert L.sphdem_create(C.byref(p), 0, 0, C.byref(h)) == -1
    q = p.copy()
    q.solver_type = 2          # DFSPH: commented out in the reference driver (SOPHIA_gpu.cu:160-162)
    assert L.sphdem_create(C.byref(q), 10, 0, C.byref(h)) == -7
    # switches of the ISPH step that are not built: property tables, the
    # Boussinesq term and the wall velocity condition
    for k in ("prop_table", "boussinesq_solve", "noslip_bc", "penetration_solve"):
        q = p.copy()
        setattr(q, k, 1)
        assert L.sphdem_create(C.byref(q), 10, 0, C.byref(h)) == -7, k
    q = p.copy()
    q.turbulence_model = 5
    assert L.sphdem_create(C.byref(q), 10, 0, C.byref(h)) == -1
    assert L.sphdem_step(None, 1) == -1
    assert L.sphdem_get_stats(None, None) == -1
    for code in (0, -1, -2, -3, -4, -5, -6, -7, -8):
        assert L.sphdem_strerror(code)


def test_params_dict_roundtrip():
    """SphdemParams survive as_dict -> JSON -> from_dict (the golden fixtures
    and the generator's params.json keep parameters by name)."""
    import json

    from fluidized_bed_master_b200.params import PRECOND_TWO_LEVEL, SphdemParams, reference_params

    p = reference_params()
    p.ppe_precond = PRECOND_TWO_LEVEL
    p.dem_list_cap = 40
    p.margin[3] = 0.125
    q = SphdemParams.from_dict(json.loads(json.dumps(p.as_dict())))
    assert bytes(q) == bytes(p)
    # fields a dictionary does not name stay zero
    r = SphdemParams.from_dict({"kappa": 2.0})
    assert r.kappa == 2.0 and r.ppe_precond == 0 and r.dem_list_cap == 0
