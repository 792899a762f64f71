"""The C ABI library loads without a GPU and exports every declared function."""
import ctypes as C
import os
import re

import conftest

ROOT = conftest.ROOT


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        if 'extern "C"' not in text:
            continue  # C++-only headers (cbm_rng.h) declare inline functions, not exports
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(cbm_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = declared_functions()
    for core in ("cbm_create", "cbm_upload", "cbm_step", "cbm_download", "cbm_destroy",
                 "cbm_get_neighbors", "cbm_get_grid", "cbm_last_error"):
        assert core in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(conftest.cbm._abi.LIB_PATH)  # no CUDA call is made
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    lib.cbm_version.restype = C.c_char_p
    assert lib.cbm_version().startswith(b"cbm_b200")


def test_create_without_device_fails_loudly():
    """On a machine without a CUDA device cbm_create returns an error (no CPU fallback)."""
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    abi = conftest.cbm._abi
    with pytest.raises(abi.CbmError):
        conftest.cbm.Context(abi.make_config(dims=2, n_max=4, box_hi=(1, 1), dt=0.1))


def test_create_rejects_capacities_beyond_the_fate_scan():
    """Births and deaths pack two prefix counts of up to 2 n_max into 29 bits
    each, so cbm_create refuses n_max >= 2^28 with a fate rule.  The argument
    check comes before any CUDA call, so it runs without a GPU."""
    import ctypes as C2
    abi = conftest.cbm._abi
    lib = abi.load_library()
    cfg = abi.make_config(dims=3, n_max=1 << 28, box_hi=(1, 1, 1), dt=0.1, fate=abi.FATE_VOLUME,
                          growth=1, v_div=2.0)
    h = C2.c_void_p()
    rc = lib.cbm_create(C2.byref(h), C2.byref(cfg))
    assert rc == 1  # CBM_ERR_ARG
    assert b"2^28" in lib.cbm_last_error(None)


def test_rods_create_rejects_bad_configurations():
    """cbm_rods_create checks its configuration before any CUDA call."""
    import pytest
    abi = conftest.cbm._abi
    base = dict(n_max=8, box_lo=(-5.0, -5.0), box_hi=(5.0, 5.0), dt=1e-4, kn=1.0, gamma_n=1.0,
                gamma_t=1.0, mu_cc=0.1, beta=0.8, beta_w=0.8, cell_edge=3.0)
    bad = [dict(neighbors=abi.NEIGH_VERLET_DISPLACEMENT), dict(neighbors=abi.NEIGH_NONE),
           dict(cell_edge=0.0), dict(dt=0.0), dict(n_max=0), dict(box_hi=(-5.0, 5.0)),
           dict(precision=7)]
    for change in bad:
        kw = dict(base, **change)
        with pytest.raises(abi.CbmError) as e:
            abi.Rods2D(abi.make_rods_config(**kw))
        assert e.value.code == abi.CBM_ERR_ARG, change


def test_rods_growth_config_checked():
    import pytest
    abi = conftest.cbm._abi
    base = dict(n_max=8, box_lo=(-5.0, -5.0), box_hi=(5.0, 5.0), dt=1e-4, kn=1.0, gamma_n=1.0,
                gamma_t=1.0, mu_cc=0.1, beta=0.8, beta_w=0.8, cell_edge=3.0)
    cfg = abi.make_rods_config(**base, growth=float("nan"), l_max=3.0)
    with pytest.raises(abi.CbmError) as e:
        abi.Rods2D(cfg)
    assert e.value.code == abi.CBM_ERR_ARG
    cfg = abi.make_rods_config(**base)
    cfg.growth_model = 2
    with pytest.raises(abi.CbmError) as e:
        abi.Rods2D(cfg)
    assert e.value.code == abi.CBM_ERR_ARG
