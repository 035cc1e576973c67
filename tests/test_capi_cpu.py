"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares with the ctypes signatures the host mirror uses, and parses
EOTArgs settings like read_args_json (Utilities.jl:18-31, 88-92)."""
import ctypes as C
import math
import os
import re

import pytest

from culamp_b200 import _lib
from culamp_b200.args import EOTArgs, args_from_json_string, default_args, read_args_json


def header_functions():
    text = open(_lib.HEADER_PATH).read()
    return sorted(set(re.findall(r"\b(culamp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), "ctypes table out of sync with culamp.h"


def test_version_and_status_strings():
    lib = _lib.load()
    assert lib.culamp_version() == 100
    assert lib.culamp_status_string(0) == b"ok"
    assert b"invalid" in lib.culamp_status_string(1)


def test_defaults_match_eotargs():
    a = default_args()
    assert a == EOTArgs()
    assert a.B == 1.0 and a.alpha == 0.01 and a.itermax == 10_000 and math.isinf(a.tmax)


def test_json_settings_like_reference_configs(tmp_path):
    # same keys / values layout as the reference's configurations/*.json
    text = """{
        "eta_p": 1e-3,
        "eta_mu": 0.0,
        "tau_p": 1.0,
        "tau_mu": 1.0,
        "alpha": 0.01,
        "B": 1.1,
        "epsilon": 1e-10,
        "itermax": 1000000,
        "verbose": true,
        "tmax": 600,
        "inner_iter": 10
    }"""
    f = tmp_path / "default_1e-03.json"
    f.write_text(text)
    a = read_args_json(str(f))
    assert a.eta_p == 1e-3 and a.B == 1.1 and a.epsilon == 1e-10
    assert a.itermax == 1_000_000 and a.tmax == 600 and a.verbose is True
    assert a.anneal_mult == 0.95   # missing key keeps its default


def test_json_partial_and_unknown_keys():
    a = args_from_json_string('{"eta_p": 0.000, "anneal_mult": 0.79370052598, "note": "x", '
                              '"nested": {"a": [1, 2]}, "verbose": false}')
    assert a.eta_p == 0.0 and a.anneal_mult == 0.79370052598 and a.verbose is False


@pytest.mark.parametrize("bad", ['{"itermax": 1.5}', '[1,2]', '{"eta_p": }', '{"eta_p" 1}'])
def test_json_rejects_malformed(bad):
    with pytest.raises(_lib.CulampError):
        args_from_json_string(bad)


def test_missing_settings_file_is_io_error(tmp_path):
    with pytest.raises(_lib.CulampError) as e:
        read_args_json(str(tmp_path / "missing.json"))
    assert e.value.status == _lib.ERR_IO


def test_create_without_gpu_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    lib = _lib.load()
    h = C.c_void_p()
    st = lib.culamp_create(C.byref(h), 0)
    assert st != 0 and not h.value
