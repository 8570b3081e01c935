"""The C-ABI library loads, exports every symbol include/b3g.h declares, and
fails loudly (no CPU fallback) where there is no GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "b3g.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(b3g_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header(b3g):
    L = C.CDLL(b3g.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings(b3g):
    L = b3g.lib()
    for s in range(10):
        assert L.b3g_status_string(s)


def test_invalid_arguments_without_device(b3g):
    L = b3g.lib()
    h = C.c_void_p()
    assert L.b3g_cloth_create(None, None, 0, C.byref(h)) == 1
    assert L.b3g_cloth_destroy(None) == 1
    assert L.b3g_cloth_step(None, 0.01, 8, 2, None) == 1
    assert L.b3g_cloth_set_assembly(None, 0) == 1
    assert L.b3g_cloth_get_assembly(None) == 1  # B3G_ASSEMBLY_ROWS for no cloth


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is not None and
                    os.environ.get("CUDA_VISIBLE_DEVICES") != "", reason="device visible")
def test_no_cpu_fallback(b3g):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    scene = b3g.plain_scene(8)
    with pytest.raises(b3g.B3gError) as e:
        b3g.Cloth(scene.mesh, scene.cdef)
    assert e.value.status == 3  # B3G_ERR_NO_DEVICE
