"""The C-ABI library loads on a machine without a GPU and exports every
function that include/*.h declares; calls that need no device behave."""
import ctypes as C
import os
import re

import pytest

import dsmsgt

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(REPO, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dsm_\w+)\s*\(", text)) - {"dsm_ctx_t"})


@pytest.mark.parametrize("header", ["dsmsgt.h", "dsmsgt_host.h"])
def test_library_exports_every_declared_function(built, header):
    L = C.CDLL(dsmsgt.LIB_PATH)
    names = declared(header)
    assert len(names) >= 5
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version_and_error_strings(built):
    L = dsmsgt.lib()
    assert L.dsm_abi_version() == 3
    for code in range(0, 8):
        s = L.dsm_strerror(code)
        assert s and len(s) >= 2
    assert L.dsm_strerror(99)


def test_no_device_is_an_error_not_a_crash(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    s = dsmsgt.Setup(__import__("cases").sh_small(), "sh")
    with pytest.raises(dsmsgt.DsmError, match="no CUDA device|DSM_ERR|failed"):
        dsmsgt.Context(s)
