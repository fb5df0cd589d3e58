"""The engine's C-ABI library loads and exports every entry point include/*.h declares."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

from finoptions import _abi

HEADERS = sorted((Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def declared_functions() -> set[str]:
    names: set[str] = set()
    for header in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names.update(re.findall(r"^\s*(?:int|void)\s+(fo_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_entry_point() -> None:
    lib = _abi.load()
    declared = declared_functions()
    assert len(declared) >= 20
    missing = [name for name in sorted(declared) if not hasattr(lib, name)]
    assert missing == []
    assert set(_abi.EXPORTED_SYMBOLS) <= declared


def test_build_info_names_the_architecture() -> None:
    buf = ctypes.create_string_buffer(256)
    assert _abi.load().fo_build_info(buf, len(buf)) == 0
    assert b"sm_100a" in buf.value


def test_struct_layouts_match_the_header_field_order() -> None:
    text = (Path(__file__).resolve().parents[1] / "include" / "finoptions_cuda.h").read_text()
    for struct, cls in (("fo_lsm_call_request", _abi.FoLsmCallRequest), ("fo_lsm_grouped_request", _abi.FoLsmGroupedRequest),
                        ("fo_gbm_seeded_request", _abi.FoGbmSeededRequest), ("fo_batch_result_columns", _abi.FoBatchResultColumns),
                        ("fo_lsm_node_diagnostic", _abi.FoLsmNodeDiagnostic), ("fo_lsm_call_result", _abi.FoLsmCallResult),
                        ("fo_lsm_call_greeks", _abi.FoLsmCallGreeks)):
        body = text[text.index(f"typedef struct {struct} {{"):]
        body = re.sub(r"/\*.*?\*/", "", body[: body.index("}")], flags=re.S)
        names = re.findall(r"\*?\s*(\w+)\s*;", body)
        names = [n for n in re.findall(r"(\w+)\s*[;,]", body) if not n.isupper()]
        assert [f[0] for f in cls._fields_] == names, struct


def test_cuda_executor_fails_loudly_without_a_device_or_opens_one() -> None:
    err = _abi.FoError()
    handle = ctypes.c_void_p()
    status = _abi.load().fo_cuda_executor_create(0, ctypes.byref(handle), ctypes.byref(err))
    if status == 0:
        _abi.load().fo_executor_destroy(handle)
    else:
        assert status == _abi.FO_ERR_EXECUTION
        assert b"no CPU fallback" in err.message or b"sm_100" in err.message
