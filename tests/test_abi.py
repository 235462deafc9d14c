"""CPU checks of the C ABI boundary, with no device call: the library loads, it
exports every function include/hs_b200.h declares, the Python binding gives each
one a signature, and the binding's constants match the header's enums."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "hs_b200.h"


@pytest.fixture(scope="module")
def header_text():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _declared_functions(text):
    pat = r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(hs_[a-z0-9_]+)\s*\("
    return sorted(set(re.findall(pat, text, flags=re.M)))


def _enum(text, name):
    body = re.search(r"typedef enum %s \{(.*?)\}" % name, text, flags=re.S).group(1)
    return {k: int(v) for k, v in re.findall(r"(HS_[A-Z0-9_]+)\s*=\s*(\d+)", body)}


def test_every_declared_function_is_exported_and_bound(hs, header_text):
    names = _declared_functions(header_text)
    assert len(names) >= 40, names
    lib = hs._lib.load()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared in hs_b200.h but not exported: {missing}"
    unbound = [n for n in names if n not in hs._lib.SIGNATURES]
    assert not unbound, f"exported but without a ctypes signature: {unbound}"
    stale = [n for n in hs._lib.SIGNATURES if n not in names]
    assert not stale, f"bound in Python but not declared in hs_b200.h: {stale}"


def test_abi_version(hs, header_text):
    v = int(re.search(r"#define HS_B200_ABI_VERSION (\d+)", HEADER.read_text()).group(1))
    assert hs._lib.load().hs_abi_version() == v == hs._lib.ABI_VERSION


def test_status_codes_and_strings(hs, header_text):
    status = _enum(header_text, "hs_status")
    assert {v: k for k, v in status.items()} == hs._lib.STATUS_NAMES
    lib = hs._lib.load()
    for code, name in hs._lib.STATUS_NAMES.items():
        assert lib.hs_status_string(code).decode() == name


def test_precision_and_kernel_ids_match_header(hs, header_text):
    prec = _enum(header_text, "hs_precision")
    assert {k: prec["HS_PRECISION_" + k.upper()] for k in hs.PRECISIONS} == hs.PRECISIONS
    assert set(prec) == {"HS_PRECISION_" + k.upper() for k in hs.PRECISIONS}
    kid = _enum(header_text, "hs_kernel_id")
    for k, v in hs._lib.KERNEL_IDS.items():
        assert kid["HS_KERNEL_" + k.upper()] == v
    assert len(hs._lib.KERNEL_IDS) == kid["HS_KERNEL_COUNT"]
