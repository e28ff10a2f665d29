"""The C-ABI library loads and exports every function include/*.h declares
(no GPU needed: nothing here calls into the device)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import slab

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# header -> the library that implements it
LIBS = {"slab_gpu.h": os.path.join(ROOT, "slab-pro_b200", "lib", "libslab_gpu.so"),
        "slab_host.h": os.path.join(ROOT, "slab-pro_b200", "lib", "libslab_sim.so")}


def declared_functions(header=None):
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        if header and os.path.basename(h) != header:
            continue
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        for m in re.finditer(r"\b(slab_[A-Za-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("slab_create", "slab_set_params", "slab_upload_particles", "slab_advance_to_frame", "slab_download_particles",
              "slab_download_grid", "slab_download_max", "slab_conservation", "slab_last_error", "slab_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        name = os.path.basename(h)
        assert name in LIBS, f"no library recorded for {name}"
        L = ctypes.CDLL(LIBS[name])
        missing = [n for n in declared_functions(name) if not hasattr(L, n)]
        assert not missing, (name, missing)


def test_version_and_status_names_without_gpu():
    L = slab.lib()
    assert b"sm_100a" in L.slab_version()
    assert L.slab_status_name(4) == b"SLAB_E_DOMAIN"


def test_null_arguments_are_rejected_without_gpu():
    L = slab.lib()
    assert L.slab_create(None, None, None) == 1
    assert b"NULL" in L.slab_last_error(None)  # a failed create leaves its message for slab_last_error(NULL)
    assert L.slab_set_params(None, None) == 1
    assert L.slab_advance_steps(None, 1, None) == 1


def test_caller_output_arrays_are_checked():
    """slab.py's caller-owned output arrays: contiguous float64 of at least
    the needed length, else ValueError before any library call."""
    a = np.zeros(10)
    assert slab._out_array(a, 8).shape == (8,)
    with pytest.raises(ValueError):
        slab._out_array(np.zeros(10, dtype=np.float32), 8)
    with pytest.raises(ValueError):
        slab._out_array(np.zeros(4), 8)
    with pytest.raises(ValueError):
        slab._out_array(np.zeros((4, 4))[:, 0], 2)
