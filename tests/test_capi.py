"""The C-ABI library: builds, loads, exports what include/dnslbm.h declares,
and rejects bad decks before touching a GPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dnslbm.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(dnslbm_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("dnslbm_create", "dnslbm_destroy", "dnslbm_step", "dnslbm_load_state", "dnslbm_store_state",
              "dnslbm_logs", "dnslbm_statistics", "dnslbm_moments", "dnslbm_set_flags"):
        assert n in names


def test_library_exports_every_declared_symbol():
    import dnslbm
    L = dnslbm.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


@pytest.mark.parametrize("kw,frag", [
    (dict(xdv=1), "too small"), (dict(zdv=2), "too small"), (dict(omega=2.5), "omega"),
    (dict(precision=8), "precision"), (dict(force_mode=7), "force mode"), (dict(bc_mode=9), "bc mode"),
])
def test_bad_deck_is_rejected_with_message(kw, frag):
    import dnslbm
    args = dict(xdv=8, ydv=8, zdv=6, omega=1.5)
    args.update(kw)
    omega = args.pop("omega")
    with pytest.raises(dnslbm.DnsLbmError) as e:
        dnslbm.Channel(args.pop("xdv"), args.pop("ydv"), args.pop("zdv"), omega, **args)
    assert e.value.code == dnslbm.ERR_ARG
    assert frag in str(e.value)
