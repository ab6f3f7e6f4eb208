"""The C-ABI library: it loads without a GPU and exports every entry point include/*.h
declares; the Python layer maps its status codes onto the reference's exceptions."""
import glob
import os
import re

import pytest

import nwgrad_b200 as nw
from nwgrad_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?\w+\s*\*?\s*(nwg_\w+)\s*\(", text, flags=re.M):
            syms.add(m.group(1))
    return syms


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ("nwg_store_create", "nwg_store_destroy", "nwg_params_set", "nwg_run", "nwg_scores",
              "nwg_grads", "nwg_reduce", "nwg_guides", "nwg_status", "nwg_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    L = nw.load_library()
    missing = [s for s in sorted(declared_symbols()) if not hasattr(L, s)]
    assert not missing, missing


def test_status_mapping():
    L = nw.load_library()
    _capi.check(_capi.NWG_OK)
    with pytest.raises(ValueError):
        _capi.check(_capi.NWG_EINVAL)
    with pytest.raises(ValueError):
        _capi.check(_capi.NWG_ERANGE)
    with pytest.raises(RuntimeError):
        _capi.check(_capi.NWG_ESTATE)
    with pytest.raises(MemoryError):
        _capi.check(_capi.NWG_ENOMEM)
    assert L.nwg_last_error() is not None
