"""CPU checks of the drop-in boundary: the library loads, exports every entry
point of include/adamantine_b200.h, and its config structure matches the
oracle's byte for byte (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from adamantine_b200 import _lib
from adamantine_b200.config import ConfigStruct, SourceStruct

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(header="adamantine_b200.h"):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"\b(adm_[A-Za-z0-9_]+)\s*\(", text)))


def all_headers():
    return sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h"))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = [n for h in all_headers() for n in header_functions(h)]
    assert len(names) >= 27
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    names = set(header_functions()) | set(header_functions("adamantine_b200_ensemble.h")) | \
        set(header_functions("adamantine_b200_adjoint.h")) | set(header_functions("adamantine_b200_deposition.h")) | \
        set(header_functions("adamantine_b200_microstructure.h")) | set(header_functions("adamantine_b200_amr.h")) | \
        set(header_functions("adamantine_b200_mechanics.h"))
    assert names - {"adm_last_error"} == set(_lib.SIGNATURES)


def test_config_layout_matches_oracle_header():
    """adm_config (include/adamantine_b200.h) and orc_config
    (oracle/thermal_oracle.h) share one layout."""
    def fields(path, struct):
        text = open(path).read()
        body = re.search(r"typedef struct %s\s*\{(.*?)\}\s*%s;" % (struct, struct), text, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        return [re.sub(r"\s+", " ", l.strip().rstrip(";")) for l in body.split(";") if l.strip()]

    a = fields(os.path.join(ROOT, "include", "adamantine_b200.h"), "adm_config")
    b = fields(os.path.join(ROOT, "oracle", "thermal_oracle.h"), "orc_config")
    norm = lambda xs: [x.replace("adm_source", "SRC").replace("orc_source", "SRC") for x in xs]
    assert norm(a) == norm(b)
    assert ctypes.sizeof(SourceStruct) == 2 * 4 + 13 * 8 + 8
    assert ConfigStruct.sources.offset % 8 == 0


def test_errors_are_reported_without_a_gpu():
    """A bad configuration is rejected on the host with a status code."""
    L = _lib.load()
    cfg = ConfigStruct()
    cfg.dim = 2  # the GPU path is 3D only
    h = ctypes.c_void_p()
    rc = L.adm_create(ctypes.byref(cfg), 0, None, ctypes.byref(h))
    assert rc != 0
    assert b"dim" in L.adm_last_error()
