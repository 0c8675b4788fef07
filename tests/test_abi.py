"""The C-ABI library loads and exports every entry point declared in include/luz_gpu.h."""
import os
import re

import pytest

from luz_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "luz_gpu.h")).read()
    return sorted(set(re.findall(r"^int\s+(luz_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "luz_gpu_render" in names and "luz_gpu_trace_rays" in names and len(names) >= 14


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared()) == set(native.EXPORTED)


def test_device_count_without_gpu_is_not_an_error():
    assert native.device_count() >= 0


def test_last_error_after_invalid_call():
    with pytest.raises(native.LuzError) as e:
        native.Pack(type("B", (), {"ptr": lambda self: None, "scene": None})())
    assert e.value.code == -1
